// Cell-tile exact kNN: the queries of one grid cell are searched together,
// one query per lane, over the cell's 3x3x3 block of candidates, which is
// staged 16 at a time in shared memory.
//
// The reference's ring search (GridKNNCuda.cu:647-743, driven level by level
// from :2322-2634) visits, for a query of level-L cell C, the points of the
// 3x3x3 block of level-L cells around C -- the same block for every query of
// C.  k_knn_plain runs one query per warp and spends ~16 warp instructions
// per candidate locating, loading and merging it.  Here each half of a warp
// takes a cell (a unit) and up to 16 of its queries, one per lane; every
// candidate of the block is loaded once per half-warp and compared by all
// of its lanes at once:
//
//   pass 1  each lane buckets its candidate distances (64 buckets, 8 per
//           octave of d^2 from (h/4)^2 to (4h)^2, h the level's cell side)
//           and finds the bucket b* holding its (k+1)-th smallest; the half
//           records the smallest bucket of each group of steps;
//   pass 2  each lane keeps the block positions (16 bits) of buckets <= b*
//           (at most tile_cap) in bucket order (offsets from pass 1's counts),
//           visiting only the step groups whose smallest bucket is at most
//           the half's largest b*; the kept distances are computed again into
//           the spent bucket space and the list is insertion-sorted (only
//           candidates of one bucket are out of order).
//
// The result is accepted only when it provably equals the ring search's list
// (the conditions of the proposal-driven box search, knn.cu): the k+1
// smallest distances are pairwise distinct; the ball of the k-th distance
// (plus a margin) lies inside the searched block, so the k kept points are
// the k nearest of the cloud; the ring search's stop step, replayed with
// decide() on that distance, visits them all; and no cell of the levels it
// visits holds max_points_in_cell points or more.  Queries whose blocks never
// reach the population that selects a level run the ring search (k_knn_plain's
// code) at the start of the same kernel; queries that fail the checks run it
// afterwards (k_knn_plain over the list of those queries).
//
// The level of a query is the first whose block around the query's cell
// holds at least kTileAlpha * (k+1) points (k_tile_assign); every cell that
// has queries at its level becomes one unit of work.
#pragma once
#include <map>
#include <mutex>
#include "knn_search.cuh"
#include "proposal.cuh"

namespace egt {
namespace {

constexpr int kTileWarps = 1;    // warps per block (one: blocks pack the SM's shared memory tightly)
constexpr int kTileBins = 64;    // distance buckets per query: 8 per octave of d^2, (h/4)^2 to (4h)^2
// S: list registers of the in-kernel ring search (k+1 <= 32 S); it also sets
// the candidates kept per query (the buckets up to b*, the query included).
template <int S>
constexpr int tile_cap() { return S <= 2 ? 64 : 96; }
constexpr int kTileMinK = 16;    // smaller k: the ring search (measured faster there)
constexpr int kTileMaxK = 64;    // largest k the cell-tile search takes
constexpr int kTileMaxK2 = 40;   // largest k of the narrower form (S = 2, 64 kept candidates)
constexpr int kTileAlpha = 6;    // block population that selects a level, in units of k+1 (measured on
                                 // 4M superquadrics at k = 40, with the sparse rule below: 5 to 7 within
                                 // 2 %, 4 and 8 slower)
constexpr int kTileSparse = 2;       // a finer block below (k+1)/kTileSparse points: the ring search (measured
                                      // on 4M superquadrics at k = 40: (k+1)/2 and 0.6(k+1) best, 0.75(k+1)
                                      // 8 % slower, 0.45(k+1) and below 15 % slower: its long searches return)
constexpr int kTileMaxBlock = 6144;   // larger blocks: the ring search (one warp would hold the search's end)
constexpr int kTileStartLevel = 3;   // the assignment's first level (the usual one on dense clouds)
constexpr int kTileClasses = 6;       // batch classes by block size (>= 4096, 2048, 1024, 512, 256, less)

struct TileArgs {
    uint8_t* lq;                      // [n] level each query is searched at (0xff: ring search)
    uint32_t* unit_bits;              // [kMaxLevels][words] cells that already have a unit
    int words;                        // words per level
    unsigned long long* units;        // [n] cloud << 40 | level << 32 | cell index
    unsigned long long* n_units;      // units written by k_tile_assign
    unsigned long long* unit_work;    // next unit to claim
    int* ring;                        // [n] queries for the ring search
    unsigned long long* n_ring;       // their count
    int maxblock;                     // kTileMaxBlock
    uint32_t* qarr;                   // [n] the units' queries, grouped by unit (k_tile_gather)
    unsigned long long* n_q;          // queries written to qarr
    uint2* batch;                     // [bcap] (unit index, first query in qarr), largest blocks first
    uint8_t* bcnt;                    // [bcap] queries in each batch (1..16)
    int bcap;                         // n + n/16 + 1 >= units + queries/16
    uint32_t* ucnt;                   // [n] queries of each unit
    uint8_t* ucls;                    // [n] class of each unit's block
    unsigned long long* cls_n;        // [kTileClasses] batches per class
    unsigned long long* cls_fill;     // [kTileClasses] batches written per class
    int* ring2;                       // [n] queries the tile search could not certify
    unsigned long long* n_ring2;      // their count
    unsigned long long* ring_work;    // next query of `ring` for the tile kernel's ring search
    // Several clouds (egt_batch): the search arguments of each cloud, and each
    // point's cloud.  Queries, lq and the ring lists then use indices over
    // all clouds' points; a single cloud passes its own arguments instead.
    const KnnArgs* desc;
    const uint16_t* cloud_of;
    int npts;                         // points of all clouds
};

// The search arguments of cloud c: the kernel's own (one cloud), or the
// cloud's descriptor.
template <bool kBatch>
__device__ __forceinline__ const KnnArgs& tile_args(const KnnArgs& a, const TileArgs& t, int c) {
    if constexpr (kBatch) return t.desc[c];
    else return a;
}

__device__ __forceinline__ unsigned long long unit_code(int c, int l, int ci) {
    return ((unsigned long long)c << 40) | ((unsigned long long)l << 32) | (unsigned)ci;
}
__device__ __forceinline__ void unit_parts(unsigned long long code, int& c, int& l, int& ci) {
    c = (int)(code >> 40);
    l = (int)((code >> 32) & 0xffu);
    ci = (int)(code & 0xffffffffu);
}

// Shared memory of one warp (both halves).
// Rows of the bucket space: the buckets, then the kept candidates' distances
// (one row each, up to tile_cap).
template <int S>
constexpr int tile_rows() { return kTileBins > tile_cap<S>() ? kTileBins : tile_cap<S>(); }

template <int S>
constexpr size_t tile_warp_bytes() {
    return (size_t)tile_rows<S>() * 32 * 4         // bucket counts, offsets, then kept distances [row][lane]
           + (size_t)tile_cap<S>() * 32 * 2        // kept candidates' block positions [slot][lane]
           + 2 * 16 * 16                           // staged candidates per half (x, y, z, point)
           + 2 * 2 * 16 * 4;                       // per half: range sequence scratch at unit set-up,
                                                   // then the step groups' smallest buckets
}

// Kept-candidate slot s of lane `lane` (16-bit entries: two lanes per bank word).
__device__ __forceinline__ int tile_slot(int s, int lane) { return s * 32 + lane; }

// Index of level cell (cx, cy, cz) in the level's cell arrays (-1: empty).
__device__ __forceinline__ int cell_index(const LevelDev& L, int cx, int cy, int cz) {
    if (cx < 0 || cx >= L.B || cy < 0 || cy >= L.B || cz < 0 || cz >= L.B) return -1;
    const int2 rr = L.row_range[cy + cz * L.B];
    int lo = rr.x, hi = rr.y;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (L.cell_x[mid] < cx) lo = mid + 1;
        else hi = mid;
    }
    return (lo < rr.y && L.cell_x[lo] == cx) ? lo : -1;
}

// Appends the flagged values of the warp to a device list (one atomic per warp).
__device__ __forceinline__ void warp_append(bool flag, uint32_t v, uint32_t* list, unsigned long long* count,
                                            int lane) {
    const unsigned m = __ballot_sync(0xffffffffu, flag);
    if (!m) return;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (flag) list[base + __popc(m & ((1u << lane) - 1u))] = v;
}

__device__ __forceinline__ void warp_append64(bool flag, unsigned long long v, unsigned long long* list,
                                              unsigned long long* count, int lane) {
    const unsigned m = __ballot_sync(0xffffffffu, flag);
    if (!m) return;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (flag) list[base + __popc(m & ((1u << lane) - 1u))] = v;
}

// Level and unit of every query; queries that no level selects (or every
// query when the admission threshold can cut lists, or when k is outside
// [kTileMinK, kTileMaxK]) go to the ring search.  i runs over the points of
// all clouds (their sorted order).
template <bool kBatch>
__global__ void __launch_bounds__(256) k_tile_assign(KnnArgs a, TileArgs t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool in = i < t.npts;
    const int c = (kBatch && in) ? (int)t.cloud_of[i] : 0;
    const KnnArgs& A = tile_args<kBatch>(a, t, c);
    const int q = i - (int)A.gbase;
    int lsel = -1, ci = -1;
    // thres > 4 exceeds every squared distance of the unit cube: all admitted
    if (in && A.k >= kTileMinK && A.k <= kTileMaxK && A.np->thres > 4.0f) {
        const int thr = kTileAlpha * (A.k + 1), sparse = (A.k + 1) / kTileSparse;
        const uint32_t c0 = __float_as_uint(A.p4[q].w);
        const int cx0 = c0 & 1023u, cy0 = (c0 >> 10) & 1023u, cz0 = (c0 >> 20) & 1023u;
        // Population of the block of level l around the query's cell; the
        // blocks are nested, so it grows with l, and the first level that
        // reaches thr is found from a start near the usual one.
        auto block_pop = [&](int l) {
            const LevelDev& LV = A.lv[l];
            const int cx = cx0 >> l, cy = cy0 >> l, cz = cz0 >> l;
            int pop = 0;
#pragma unroll
            for (int r = 0; r < 9; r++) {
                const int2 g = row_points(LV, cx - 1, cx + 1, cy + r % 3 - 1, cz + r / 3 - 1);
                pop += g.y - g.x;
            }
            return pop;
        };
        int l = kTileStartLevel, pop = block_pop(l), prev = INT_MAX;  // prev: the block one level finer
        if (pop >= thr) {
            while (l > 0) {
                const int below = block_pop(l - 1);
                if (below < thr) { prev = below; break; }
                l--;
                pop = below;
            }
        } else {
            while (l + 1 < kMaxLevels && pop < thr) {
                prev = pop;
                pop = block_pop(++l);
            }
        }
        if (pop >= thr) {
            // kMaxLevels: a block too large, or a query alone in its finer
            // block -- the ring search (such a query's k nearest lie far
            // off, beyond the block, and its search climbs high)
            lsel = pop <= t.maxblock && prev >= sparse ? l : kMaxLevels;
            if (lsel == l) ci = cell_index(A.lv[l], cx0 >> l, cy0 >> l, cz0 >> l);
        }
    }
    if (lsel >= kMaxLevels || ci < 0) lsel = -1;  // ci < 0 cannot happen: the query's own cell is occupied
    // The tile kernel runs the ring search of the queries its k range takes
    // but no level selects (few, some long: they overlap the batches); the
    // clouds outside that range run it in the launch after the tile kernel,
    // at the ring search's own occupancy.
    const bool ring = in && lsel < 0;
    const bool early = A.k >= kTileMinK && A.k <= kTileMaxK;
    warp_append(ring && early, (uint32_t)i, reinterpret_cast<uint32_t*>(t.ring), t.n_ring, lane);
    warp_append(ring && !early, (uint32_t)i, reinterpret_cast<uint32_t*>(t.ring2), t.n_ring2, lane);
    if (in) t.lq[i] = lsel < 0 ? (uint8_t)0xff : (uint8_t)lsel;
    bool fresh = false;
    if (lsel >= 0) {
        // a cell is named by the first position of its points in the level's order
        const int first = (int)A.gbase + A.lv[lsel].cell_start[ci];
        const uint32_t bit = 1u << (first & 31);
        fresh = !(atomicOr(t.unit_bits + (size_t)lsel * t.words + (first >> 5), bit) & bit);
    }
    warp_append64(fresh, unit_code(c, lsel, ci), t.units, t.n_units, lane);
}

// Class of a block of `pop` candidates: larger blocks are searched first, and
// batches claimed together have blocks of similar size (the two halves of a
// warp run in step, each as long as the larger of their blocks).
__device__ __forceinline__ int tile_class(int pop) {
    return pop >= 4096 ? 0 : pop >= 2048 ? 1 : pop >= 1024 ? 2 : pop >= 512 ? 3 : pop >= 256 ? 4 : 5;
}

// Per unit (one warp per unit, grid-stride): its query count and block class,
// and the batch count of each class.
template <bool kBatch>
__global__ void __launch_bounds__(256) k_tile_count(KnnArgs a, TileArgs t) {
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)((gridDim.x * blockDim.x) >> 5);
    const unsigned long long nu = *t.n_units;
    for (unsigned long long u = gw; u < nu; u += nw) {
        int c, l, ci;
        unit_parts(t.units[u], c, l, ci);
        const KnnArgs& A = tile_args<kBatch>(a, t, c);
        const LevelDev& LV = A.lv[l];
        const int* order = l ? LV.order : nullptr;
        const int cs = LV.cell_start[ci], ce = LV.cell_start[ci + 1];
        const uint8_t* lq = t.lq + A.gbase;
        int cnt = 0;
        for (int s = cs; s < ce; s += 32) {
            bool sel = false;
            if (s + lane < ce) {
                const int qq = order ? order[s + lane] : s + lane;
                sel = lq[qq] == (uint8_t)l;
            }
            cnt += __popc(__ballot_sync(0xffffffffu, sel));
        }
        const int p0 = order ? order[cs] : cs;
        const uint32_t cc = __float_as_uint(A.p4[p0].w);
        const int cx = (int)(cc & 1023u) >> l, cy = (int)((cc >> 10) & 1023u) >> l, cz = (int)((cc >> 20) & 1023u) >> l;
        int pop = 0;
        if (lane < 9) {
            const int2 g = row_points(LV, cx - 1, cx + 1, cy + lane % 3 - 1, cz + lane / 3 - 1);
            pop = g.y - g.x;
        }
        pop = __reduce_add_sync(0xffffffffu, pop);
        const int cls = tile_class(pop);
        if (lane == 0) {
            t.ucnt[u] = (uint32_t)cnt;
            t.ucls[u] = (uint8_t)cls;
            atomicAdd(&t.cls_n[cls], (unsigned long long)((cnt + 15) >> 4));
        }
    }
}

// Compacts each unit's queries into qarr and cuts them into batches of up to
// 16 (one warp per unit, grid-stride), the batches ordered by class.
template <bool kBatch>
__global__ void __launch_bounds__(256) k_tile_gather(KnnArgs a, TileArgs t) {
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)((gridDim.x * blockDim.x) >> 5);
    const unsigned long long nu = *t.n_units;
    // first batch of each class
    unsigned long long coff = 0;
    {
        unsigned long long v = lane < kTileClasses ? t.cls_n[lane] : 0ull;
        unsigned long long incl = v;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const unsigned long long w = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += w;
        }
        coff = incl - v;
    }
    for (unsigned long long u = gw; u < nu; u += nw) {
        int c, l, ci;
        unit_parts(t.units[u], c, l, ci);
        const KnnArgs& A = tile_args<kBatch>(a, t, c);
        const LevelDev& LV = A.lv[l];
        const int* order = l ? LV.order : nullptr;
        const int cs = LV.cell_start[ci], ce = LV.cell_start[ci + 1];
        const uint8_t* lq = t.lq + A.gbase;
        const int cnt = (int)t.ucnt[u], cls = (int)t.ucls[u];
        const int nbat = (cnt + 15) >> 4;
        const unsigned long long base = __shfl_sync(0xffffffffu, coff, cls);
        unsigned long long qb = 0, bb = 0;
        if (lane == 0 && cnt > 0) {
            qb = atomicAdd(t.n_q, (unsigned long long)cnt);
            bb = base + atomicAdd(&t.cls_fill[cls], (unsigned long long)nbat);
        }
        qb = __shfl_sync(0xffffffffu, qb, 0);
        bb = __shfl_sync(0xffffffffu, bb, 0);
        int w = 0;
        for (int s = cs; s < ce && w < cnt; s += 32) {
            bool sel = false;
            int qq = -1;
            if (s + lane < ce) {
                qq = order ? order[s + lane] : s + lane;
                sel = lq[qq] == (uint8_t)l;
            }
            const unsigned m = __ballot_sync(0xffffffffu, sel);
            if (sel) t.qarr[qb + w + __popc(m & ((1u << lane) - 1u))] = (uint32_t)qq;
            w += __popc(m);
        }
        for (int j = lane; j < nbat; j += 32) {
            t.batch[bb + j] = make_uint2((uint32_t)u, (uint32_t)(qb + 16 * j));
            t.bcnt[bb + j] = (uint8_t)min(16, cnt - 16 * j);
        }
    }
}

// Half-warp form of range_seq (knn_search.cuh): the ranges of a half's lanes
// (hl = lane within the half, hf = which half) as one flattened sequence.
// All 32 lanes call it; each half gets its own sequence.
__device__ __forceinline__ RangeSeq range_seq16(int sz, int cs, int hl, int hf, int* s_pref, int* s_start) {
    int incl = sz;
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o, 16);
        if (hl >= o) incl += v;
    }
    const unsigned ne = (__ballot_sync(0xffffffffu, sz > 0) >> (16 * hf)) & 0xffffu;
    RangeSeq q;
    q.total = __shfl_sync(0xffffffffu, incl, 15, 16);
    q.m = __popc(ne);
    __syncwarp();
    if (sz > 0) {
        const int r = __popc(ne & ((1u << hl) - 1u));
        s_pref[r] = incl;
        s_start[r] = cs;
    }
    __syncwarp();
    q.incl = hl < q.m ? s_pref[hl] : INT_MAX;
    q.cs = hl < q.m ? s_start[hl] : 0;
    __syncwarp();
    return q;
}

// Half-warp form of seq_index: point index of candidate base + hl of the
// half's sequence (-1 past its end).  All 32 lanes call it.
__device__ __forceinline__ int seq_index16(const RangeSeq& q, int base, int hl, int hf,
                                           const int* __restrict__ order) {
    const int before = __popc((__ballot_sync(0xffffffffu, q.incl <= base) >> (16 * hf)) & 0xffffu);
    const int at = q.incl - base;
    const unsigned sb = (at > 0 && at < 16) ? (1u << at) : 0u;
    const unsigned starts = (__reduce_or_sync(0xffffffffu, sb << (16 * hf)) >> (16 * hf)) & 0xffffu;
    const int c = before + __popc(starts & ((2u << hl) - 1u));
    const int prev_end = __shfl_sync(0xffffffffu, q.incl, (c - 1) & 15, 16);
    const int cs = __shfl_sync(0xffffffffu, q.cs, c & 15, 16);
    const int j = base + hl;
    if (j >= q.total) return -1;
    const int pos = cs + (j - (c > 0 ? prev_end : 0));
    return order ? __ldg(order + pos) : pos;
}

__device__ __forceinline__ uint32_t tile_bin(float d, uint32_t lo) {
    return min((max(__float_as_uint(d), lo) - lo) >> 20, (uint32_t)(kTileBins - 1));
}

// State of one half-warp's current unit (uniform within the half).
struct TileUnit {
    RangeSeq seq;
    const int* order;
    uint32_t lo;   // float bits of the lower edge of bucket 1 less one bucket
    int l;         // level; -1 = no unit
    // the block's ranges r < seq.m: pref[r] = inclusive prefix end of range r
    // (INT_MAX past the last), adj[r] = its start less the positions before it
    int pref[8], adj[9];
};

// Point index of block position `pos` of a half's unit: position pos lies in
// range r, the number of ranges ending at or before it, and its level-order
// slot is pos + adj[r] (the prefix ends increase, so the last test that holds
// picks r).
__device__ __forceinline__ int tile_point(int pos, const TileUnit& U) {
    int a = U.adj[0];
#pragma unroll
    for (int t = 0; t < 8; t++) a = pos >= U.pref[t] ? U.adj[t + 1] : a;
    const int local = pos + a;
    return U.order ? __ldg(U.order + local) : local;
}

// Streams both halves' blocks through their staging buffers, 16 candidates
// per half at a time, calling f(s) for step s: the half's staged candidates
// are the block positions 16 s .. 16 s + 15 (padding past a block's end lies
// far away with index -1).
template <typename F>
__device__ __forceinline__ void tile_stream16(const TileUnit& U, bool live, int steps, const float4* __restrict__ p4,
                                              float4* chunk, int hl, int hf, F&& f) {
    const float4 far = make_float4(1e18f, 1e18f, 1e18f, 0.f);
    // software pipeline: the point index of step s+2 and the position of
    // step s+1 are in flight while step s is compared
    int pB = seq_index16(U.seq, 0, hl, hf, U.order);
    int pA = seq_index16(U.seq, 16, hl, hf, U.order);
    if (!live) pA = pB = -1;
    float4 vB = pB >= 0 ? __ldg(p4 + pB) : far;
    for (int s = 0; s < steps; s++) {
        __syncwarp();
        chunk[hl] = make_float4(vB.x, vB.y, vB.z, __int_as_float(pB));
        __syncwarp();
        pB = pA;
        vB = pB >= 0 ? __ldg(p4 + pB) : far;
        pA = seq_index16(U.seq, (s + 2) * 16, hl, hf, U.order);
        if (!live) pA = -1;
        f(s);
    }
    __syncwarp();
}

// The same stream over a sequence of steps of each half's own: s0 its first
// step, nxt(s) the step after s (a value >= end: none left).  The warp runs
// until both halves are done; a half that is done stages padding.
template <typename N, typename F>
__device__ __forceinline__ void tile_stream16_seq(const TileUnit& U, int s0, int end, N&& nxt,
                                                  const float4* __restrict__ p4, float4* chunk, int hl, int hf,
                                                  F&& f) {
    const float4 far = make_float4(1e18f, 1e18f, 1e18f, 0.f);
    int s1 = nxt(s0), s2 = nxt(s1);
    int pB = seq_index16(U.seq, min(s0, end) * 16, hl, hf, U.order);
    int pA = seq_index16(U.seq, min(s1, end) * 16, hl, hf, U.order);
    if (s0 >= end) pB = -1;
    if (s1 >= end) pA = -1;
    float4 vB = pB >= 0 ? __ldg(p4 + pB) : far;
    while (__any_sync(0xffffffffu, s0 < end)) {
        __syncwarp();
        chunk[hl] = make_float4(vB.x, vB.y, vB.z, __int_as_float(pB));
        __syncwarp();
        pB = pA;
        vB = pB >= 0 ? __ldg(p4 + pB) : far;
        pA = seq_index16(U.seq, min(s2, end) * 16, hl, hf, U.order);
        if (s2 >= end) pA = -1;
        f(s0);
        s0 = s1;
        s1 = s2;
        s2 = nxt(s2);
    }
    __syncwarp();
}

// Sets up a new unit for the lanes with `take` (both halves call it; a half
// with take = false keeps its unit).
__device__ __forceinline__ void tile_unit_setup(const KnnArgs& a, const NormParams& np, int l, int ci, bool take,
                                                int hl, int hf, int* s_pref, int* s_start, TileUnit& U) {
    int2 rg = make_int2(0, 0);
    int cx = 0, cy = 0, cz = 0;
    const int* order = nullptr;
    if (take) {
        const LevelDev& LV = a.lv[l];
        order = l ? LV.order : nullptr;
        const int cs = LV.cell_start[ci];
        const int p0 = order ? order[cs] : cs;
        const uint32_t cc = __float_as_uint(a.p4[p0].w);
        cx = (int)(cc & 1023u) >> l;
        cy = (int)((cc >> 10) & 1023u) >> l;
        cz = (int)((cc >> 20) & 1023u) >> l;
        if (hl < 9) rg = row_points(LV, cx - 1, cx + 1, cy + hl % 3 - 1, cz + hl / 3 - 1);
    }
    const RangeSeq seq = range_seq16(rg.y - rg.x, rg.x, hl, hf, s_pref, s_start);
    if (take) {
        U.seq = seq;
        U.order = order;
        U.l = l;
        int before = 0;  // positions of the ranges before range t
#pragma unroll
        for (int t = 0; t < 9; t++) {
            const bool in = t < seq.m;
            const int end = in ? s_pref[t] : INT_MAX;
            U.adj[t] = in ? s_start[t] - before : 0;
            if (t < 8) U.pref[t] = end;
            if (in) before = end;
        }
        // buckets: 8 per octave of d^2, bucket 0 below (h/4)^2 and 1/8 octave,
        // bucket kTileBins-1 from 16 h^2 up
        const float h = __fmul_rn(__fsub_rn(np.b, np.a), (float)(1 << l) * (1.0f / 1024.0f));
        U.lo = __float_as_uint(__fmul_rn(16.0f, __fmul_rn(h, h))) - ((uint32_t)(kTileBins - 1) << 20);
    }
}

// Persistent: each half-warp claims batches (up to 16 queries of one unit)
// one at a time; both halves run their batches together.
template <bool kBatch, int S>
__global__ void __launch_bounds__(kTileWarps * 32, 16) k_knn_tile(KnnArgs a, TileArgs t) {
    constexpr int kCap = tile_cap<S>();
    constexpr size_t kWarpBytes = tile_warp_bytes<S>();
    extern __shared__ __align__(16) unsigned char s_tile[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int hl = lane & 15, hf = lane >> 4;
    unsigned char* base = s_tile + (size_t)w * kWarpBytes;
    uint32_t* hist = reinterpret_cast<uint32_t*>(base);
    uint16_t* bpos = reinterpret_cast<uint16_t*>(base + (size_t)tile_rows<S>() * 32 * 4);
    float4* chunk = reinterpret_cast<float4*>(bpos + (size_t)kCap * 32) + 16 * hf;
    int* s_pref = reinterpret_cast<int*>(reinterpret_cast<float4*>(bpos + (size_t)kCap * 32) + 32) + 32 * hf;
    int* s_start = s_pref + 16;
    uint32_t* hcol = hist + lane;
    unsigned long long evals = 0;
    unsigned maxlev = 0;
    // First the ring search (k_knn_plain's code, one query per warp) of the
    // queries no level selected, while the other warps already search
    // batches, so that the long ones do not end the search.  Its scratch lies
    // in the kept-candidate space.  (Queries that fail the checks run it in a
    // separate launch at the ring kernel's own occupancy: measured faster than
    // running them here, between batches.)
    int* r_pref = reinterpret_cast<int*>(bpos);
    int* r_start = r_pref + 32;
    float* r_md = reinterpret_cast<float*>(r_start + 32);
    int* r_mp = reinterpret_cast<int*>(r_md + 32 * S);
    unsigned reruns = 0;
    auto ring_query = [&](int i) {  // i: over all clouds' points
        const int c = kBatch ? (int)t.cloud_of[i] : 0;
        const KnnArgs& A = tile_args<kBatch>(a, t, c);
        const int q = i - (int)A.gbase;
        const NormParams np = *A.np;
        WarpList<S> L;
        bool invalid, rerun;
        const int reached = plain_query<true, S>(A, np, q, A.p4[q], L, invalid, lane, r_pref, r_start, r_md, r_mp,
                                                 rerun);
        write_query<S>(A, q, L, invalid, reached, lane);
        if constexpr (kBatch) {
            if (rerun && lane == 0) atomicAdd(&A.counters[kCtrExactRerun], 1ull);
        } else {
            reruns += rerun ? 1u : 0u;
            evals += L.ev;
        }
    };
    {
        const unsigned long long n_r = *t.n_ring;
        for (;;) {
            unsigned long long j = 0;
            if (lane == 0) j = atomicAdd(t.ring_work, 1ull);
            j = __shfl_sync(0xffffffffu, j, 0);
            if (j >= n_r) break;
            ring_query(t.ring[j]);
        }
        __syncwarp();
    }
    for (int b = 0; b < kTileBins; b++) hcol[b * 32] = 0u;
    TileUnit U;
    U.seq.incl = INT_MAX;
    U.seq.cs = 0;
    U.seq.m = 0;
    U.seq.total = 0;
    U.order = nullptr;
    U.lo = 0u;
    U.l = -1;
#pragma unroll
    for (int t = 0; t < 9; t++) {
        U.adj[t] = 0;
        if (t < 8) U.pref[t] = INT_MAX;
    }
    unsigned long long n_batches = 0;
#pragma unroll
    for (int c = 0; c < kTileClasses; c++) n_batches += t.cls_n[c];
    for (;;) {
        // each half claims one batch: largest blocks first
        unsigned long long c = 0;
        if (hl == 0) c = atomicAdd(t.unit_work, 1ull);
        c = __shfl_sync(0xffffffffu, c, 16 * hf);
        const bool take = c < n_batches;
        if (!__any_sync(0xffffffffu, take)) break;
        const long long bi = take ? (long long)c : 0;
        const uint2 bd = take ? t.batch[bi] : make_uint2(0u, 0u);
        const int nq = take ? (int)t.bcnt[bi] : 0;
        int uc = 0, ul = 0, uci = 0;
        unit_parts(t.units[bd.x], uc, ul, uci);
        const KnnArgs& A = tile_args<kBatch>(a, t, uc);  // the half's cloud
        const NormParams np = *A.np;
        const int k = A.k;
        const float4* __restrict__ p4 = A.p4;
        tile_unit_setup(A, np, ul, uci, take, hl, hf, s_pref, s_start, U);
        const bool act = hl < nq;
        const int q = act ? (int)t.qarr[bd.y + hl] : -1;
        const float4 pq = act ? p4[q] : make_float4(3e18f, 3e18f, 3e18f, 0.f);
        const int total = take ? U.seq.total : 0;
        const int steps = (max(total, __shfl_xor_sync(0xffffffffu, total, 16)) + 15) >> 4;
        const uint32_t lo = U.lo;
        // The smallest bucket of each group of g steps over the half's lanes
        // (one byte per group in the half's scratch, which the unit set-up no
        // longer needs): pass 2 visits only the groups that can hold a
        // candidate it keeps.  2^gs steps per byte (128 bytes cover a block
        // of up to 8192 candidates).
        const unsigned hmask = hf ? 0xffff0000u : 0x0000ffffu;
        const int steps_h = (total + 15) >> 4;
        const int gs = steps_h > 256 ? 2 : steps_h > 128 ? 1 : 0;
        uint8_t* mb = reinterpret_cast<uint8_t*>(s_pref);
        s_pref[hl] = -1;
        s_pref[hl + 16] = -1;
        __syncwarp();
        // pass 1: bucket counts (the query itself included, at distance 0)
        tile_stream16(U, take, steps, p4, chunk, hl, hf, [&](int st) {
            uint32_t bk[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const float4 c = chunk[j];
                bk[j] = tile_bin(fs_dist3(pq.x, pq.y, pq.z, c.x, c.y, c.z), lo);
            }
#pragma unroll
            for (int j = 0; j < 16; j++) atomicAdd(hcol + bk[j] * 32, 1u);
            uint32_t mn = bk[0];
#pragma unroll
            for (int j = 1; j < 16; j++) mn = min(mn, bk[j]);
            mn = __reduce_min_sync(hmask, mn);
            if (hl == 0 && st < steps_h) {
                const int gi = st >> gs;
                mb[gi] = (uint8_t)min((uint32_t)mb[gi], mn);
            }
        });
        // bucket offsets and the bucket b* of the (k+1)-th distance other
        // than the query's own
        int cum = 0, bstar = -1, m = 0;
#pragma unroll 8
        for (int b = 0; b < kTileBins; b++) {
            const int c = (int)hcol[b * 32];
            hcol[b * 32] = (uint32_t)cum;
            cum += c;
            if (bstar < 0 && cum >= k + 2) { bstar = b; m = cum; }
        }
        bool ok = act && bstar >= 0 && bstar < kTileBins - 1 && m <= kCap;
        const float T = ok ? __uint_as_float(lo + ((uint32_t)(bstar + 1) << 20)) : 0.0f;
        // pass 2: the candidates of buckets <= b*, in bucket order, from the
        // step groups whose smallest bucket is at most the half's largest b*
        const int bmax = __reduce_max_sync(hmask, ok ? bstar : -1);
        auto nxt = [&](int st) {
            int u = st + 1;
            while (u < steps_h) {
                const int gi = u >> gs;
                if ((int)mb[gi] <= bmax) break;
                u = (gi + 1) << gs;
            }
            return min(u, steps_h);
        };
        tile_stream16_seq(U, nxt(-1), steps_h, nxt, p4, chunk, hl, hf, [&](int st) {
#pragma unroll
            for (int j0 = 0; j0 < 16; j0 += 8) {
                float dd[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const float4 c = chunk[j0 + j];
                    dd[j] = fs_dist3(pq.x, pq.y, pq.z, c.x, c.y, c.z);
                }
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    if (dd[j] < T) {
                        const uint32_t s = atomicAdd(hcol + tile_bin(dd[j], lo) * 32, 1u);
                        bpos[tile_slot((int)s, lane)] = (uint16_t)(st * 16 + j0 + j);
                    }
                }
            }
        });
        float kth = 0.0f;
        int reached = 0;
        int self = 0;  // slot of the query itself after sorting; entry i of the list is slot i + (i >= self)
        if (ok) {
            // the kept candidates' distances, into the bucket space (its offsets are spent)
#pragma unroll 4
            for (int i = 0; i < m; i++) {
                const float4 v = __ldg(p4 + tile_point(bpos[tile_slot(i, lane)], U));
                hcol[i * 32] = __float_as_uint(fs_dist3(pq.x, pq.y, pq.z, v.x, v.y, v.z));
            }
            // sorted by (distance, block position); only candidates of one bucket are out of order
            for (int i = 1; i < m; i++) {
                const uint32_t ed = hcol[i * 32], ei = bpos[tile_slot(i, lane)];
                int j = i;
                while (j > 0) {
                    const uint32_t gd = hcol[(j - 1) * 32], gi = bpos[tile_slot(j - 1, lane)];
                    if (gd < ed || (gd == ed && gi < ei)) break;
                    hcol[j * 32] = gd;
                    bpos[tile_slot(j, lane)] = (uint16_t)gi;
                    j--;
                }
                hcol[j * 32] = ed;
                bpos[tile_slot(j, lane)] = (uint16_t)ei;
            }
            // the query sits among the distance-0 entries at the front
            while (self < m - 1 && tile_point(bpos[tile_slot(self, lane)], U) != q) self++;
            // (1) the k+1 smallest distances pairwise distinct
            uint32_t prev = hcol[(self == 0 ? 1 : 0) * 32];
            for (int i = 1; i <= k && ok; i++) {
                const uint32_t cur = hcol[(i + (i >= self)) * 32];
                ok = cur != prev;
                prev = cur;
            }
        }
        if (ok) {
            const int l = U.l;
            kth = __uint_as_float(hcol[(k - 1 + (k - 1 >= self)) * 32]);
            const uint32_t c0 = __float_as_uint(pq.w);
            const int cq[3] = {(int)(c0 & 1023u), (int)((c0 >> 10) & 1023u), (int)((c0 >> 20) & 1023u)};
            // (2) the k-th ball inside the searched block
            int lo3[3], end3[3];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                lo3[d] = ((cq[d] >> l) - 1) << l;
                end3[d] = ((cq[d] >> l) + 2) << l;
            }
            ok = ball_in_box(np, pq, kth, lo3, end3);
            // (3) the ring search's stop step
            int sf = -1;
            if (ok) {
                for (int st = 0; st <= kMaxLevels; st++) {
                    const int Ls = st == 0 ? 0 : st - 1, o = st == 0 ? 0 : 1;
                    if (!decide(np, Ls, o, k, k, kth, false, pq, cq[0], cq[1], cq[2])) { sf = st; break; }
                }
                ok = sf >= 0;
            }
            if (ok) {
                const int Lf = sf == 0 ? 0 : sf - 1, of = sf == 0 ? 0 : 1;
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    lo3[d] = ((cq[d] >> Lf) - of) << Lf;
                    end3[d] = ((cq[d] >> Lf) + of + 1) << Lf;
                }
                if (!ball_in_box(np, pq, kth, lo3, end3)) {
                    for (int i = 0; i < k && ok; i++) {
                        const int p = tile_point(bpos[tile_slot(i + (i >= self), lane)], U);
                        ok = visit_step(__float_as_uint(p4[p].w), c0) <= sf;
                    }
                }
            }
            // (4) no oversized cell on the visited levels
            if (ok)
                for (int L = 0; L <= max(sf - 1, 0) && ok; L++)
                    ok = A.counters[kCtrMaxPop + L] < (unsigned long long)A.max_pts;
            reached = max(sf - 1, 0);
        }
        if (ok) {
            int* row = A.lists + (size_t)q * k;
            for (int i = 0; i < k; i++) row[i] = tile_point(bpos[tile_slot(i + (i >= self), lane)], U);
            if (A.kth_out) A.kth_out[q] = kth;
            if (A.qlevel) A.qlevel[q] = (uint8_t)reached;
            if constexpr (kBatch) {
                atomicMax(&A.counters[kCtrMaxLevel], (unsigned long long)reached);
            } else {
                maxlev = max(maxlev, (unsigned)reached);
            }
        }
        if (!kBatch && hl == 0) evals += (unsigned long long)total * nq;
        warp_append(act && !ok, (uint32_t)(A.gbase + q), reinterpret_cast<uint32_t*>(t.ring2), t.n_ring2, lane);
#pragma unroll 8
        for (int b = 0; b < kTileBins; b++) hcol[b * 32] = 0u;
    }
    if constexpr (kBatch) return;  // per-cloud counters were updated as the queries finished
    maxlev = __reduce_max_sync(0xffffffffu, maxlev);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) evals += __shfl_xor_sync(0xffffffffu, evals, o);
    if (lane == 0) {
        if (reruns) atomicAdd(&a.counters[kCtrExactRerun], (unsigned long long)reruns);
        if (evals) atomicAdd(&a.counters[kCtrEvals], evals);
        if (maxlev) atomicMax(&a.counters[kCtrMaxLevel], (unsigned long long)maxlev);
    }
}


// Working buffers of the cell-tile search for the handle's n points (all
// clouds' points for a batch), and its counters reset.
inline egt_status tile_prepare(egt_handle* h, TileArgs* t) {
    const int64_t n = h->n;
    const int words = (int)((n + 31) / 32);
    const int64_t bcap = n + n / 16 + 1;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t b_lq = al((size_t)n), b_bits = al((size_t)kMaxLevels * words * 4), b_n4 = al(4 * (size_t)n);
    const size_t b_n8 = al(8 * (size_t)n);
    const size_t b_batch = al(8 * (size_t)bcap), b_bcnt = al((size_t)bcap), b_ctr = 256;
    const size_t need = b_ctr + b_lq + b_bits + b_n8 + 4 * b_n4 + b_batch + b_bcnt + b_lq;
    if (h->tile_bytes < need) {
        dev_free(h, h->tile_mem);
        h->tile_mem = nullptr;
        h->tile_bytes = 0;
        EGT_CUDA_TRY(dev_alloc(h, &h->tile_mem, need));
        h->tile_bytes = need;
    }
    unsigned char* m = static_cast<unsigned char*>(h->tile_mem);
    unsigned long long* tctr = reinterpret_cast<unsigned long long*>(m);  // class counts and fills
    t->cls_n = tctr;
    t->cls_fill = tctr + kTileClasses;
    m += b_ctr;
    t->lq = m;
    m += b_lq;
    t->unit_bits = reinterpret_cast<uint32_t*>(m);
    m += b_bits;
    t->words = words;
    t->units = reinterpret_cast<unsigned long long*>(m);
    m += b_n8;
    t->ring = reinterpret_cast<int*>(m);
    m += b_n4;
    t->ring2 = reinterpret_cast<int*>(m);
    m += b_n4;
    t->qarr = reinterpret_cast<uint32_t*>(m);
    m += b_n4;
    t->ucnt = reinterpret_cast<uint32_t*>(m);
    m += b_n4;
    t->batch = reinterpret_cast<uint2*>(m);
    m += b_batch;
    t->bcnt = m;
    m += b_bcnt;
    t->ucls = m;
    t->bcap = (int)bcap;
    t->n_units = h->d_counters + kCtrTileUnits;
    t->unit_work = h->d_counters + kCtrTileWork;
    t->n_ring = h->d_counters + kCtrSelFallback;
    t->n_q = h->d_counters + kCtrTileQ;
    t->n_ring2 = h->d_counters + kCtrTileRing2;
    t->ring_work = h->d_counters + kCtrTileRingWork1;
    t->maxblock = kTileMaxBlock;
    t->desc = nullptr;
    t->cloud_of = nullptr;
    t->npts = (int)n;
    cudaStream_t st = h->stream;
    EGT_CUDA_TRY(cudaMemsetAsync(t->unit_bits, 0, b_bits, st));
    EGT_CUDA_TRY(cudaMemsetAsync(tctr, 0, b_ctr, st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrTileUnits, 0, 8 * sizeof(unsigned long long), st));
    return EGT_OK;
}

// Assignment, batching and the tile kernel (with the ring search of the
// queries no level selected); the uncertified queries are left in t.ring2.
template <bool kBatch, int S>
egt_status tile_kernel_launch(const KnnArgs& a, const TileArgs& t, cudaStream_t st) {
    constexpr size_t smem = tile_warp_bytes<S>() * kTileWarps;
    static std::mutex mu;
    static std::map<int, unsigned> waves;  // per device: blocks of one resident wave
    int dev = 0;
    EGT_CUDA_TRY(cudaGetDevice(&dev));
    unsigned G = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = waves.find(dev);
        if (it != waves.end()) G = it->second;
    }
    if (!G) {
        EGT_CUDA_TRY(cudaFuncSetAttribute(k_knn_tile<kBatch, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        int sms = 0, per = 0;
        EGT_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        EGT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_knn_tile<kBatch, S>, kTileWarps * 32,
                                                                    smem));
        G = (unsigned)std::max(1, sms * std::max(per, 1));
        std::lock_guard<std::mutex> lock(mu);
        waves[dev] = G;
    }
    k_knn_tile<kBatch, S><<<G, kTileWarps * 32, smem, st>>>(a, t);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

// kmax: the largest k among the queries the tile search takes.
template <bool kBatch>
egt_status tile_launch(const KnnArgs& a, const TileArgs& t, int kmax, cudaStream_t st) {
    const unsigned T = 256;
    const int64_t npts = t.npts;
    k_tile_assign<kBatch><<<(unsigned)((npts + T - 1) / T), T, 0, st>>>(a, t);
    EGT_LAUNCH_CHECK();
    const unsigned Gu = (unsigned)std::min<int64_t>(4096, (npts + T - 1) / T);
    k_tile_count<kBatch><<<Gu, T, 0, st>>>(a, t);
    EGT_LAUNCH_CHECK();
    k_tile_gather<kBatch><<<Gu, T, 0, st>>>(a, t);
    EGT_LAUNCH_CHECK();
    return kmax <= kTileMaxK2 ? tile_kernel_launch<kBatch, 2>(a, t, st) : tile_kernel_launch<kBatch, 3>(a, t, st);
}

}  // namespace
}  // namespace egt
