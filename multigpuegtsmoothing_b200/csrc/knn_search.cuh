// Device side of the exact grid kNN search, shared by the single-cloud kernels
// (knn.cu) and the batched kernels (batch.cu).  See knn.cu for the reference
// correspondence and the design.
#pragma once
#include <climits>
#include "egt_internal.cuh"
#include "knn_common.cuh"

namespace egt {
namespace {

struct KnnArgs {
    const float4* __restrict__ p4;
    const NormParams* __restrict__ np;
    LevelDev lv[kMaxLevels];
    int n, k, max_pts;
    int chunk;  // queries claimed per atomic by the persistent kernels
    int* __restrict__ lists;
    float* __restrict__ kth_out;
    uint8_t* __restrict__ qlevel;
    unsigned long long* __restrict__ counters;
    const int* __restrict__ qmap = nullptr;  // query j of a launch is qmap[j] (nullptr: j)
    unsigned long long* __restrict__ work = nullptr;  // work counter (nullptr: counters[kCtrWork])
    const unsigned long long* __restrict__ n_dev = nullptr;  // launch size on the device (nullptr: n)
    unsigned long long* __restrict__ n_ring = nullptr;  // ring-search query count (nullptr: counters[kCtrSelFallback])
    int64_t gbase = 0;  // index of the cloud's first point in a batch's point arrays
};

// Queries of a launch: n, or the count a preceding kernel left on the device.
__device__ __forceinline__ int launch_size(const KnnArgs& a) { return a.n_dev ? (int)*a.n_dev : a.n; }

constexpr int kWarps = 8;
// The search kernels are latency-bound: keep four blocks (32 warps) resident
// per SM, which caps them at 64 registers (measured faster than fewer,
// larger-register blocks for lists of up to 96 slots).
constexpr int kMinBlocks = 4;

// Continue decision after the last cube of a shell (GridKNNCuda.cu:694-741).
__device__ __forceinline__ bool decide(const NormParams& np, int L, int o, int counter, int k, float kth,
                                       bool invalid, float4 q, int cx0, int cy0, int cz0) {
    if (invalid) return false;
    const int B = 1024 >> L;
    const float h = __fdiv_rn(__fsub_rn(np.b, np.a), (float)B);
    const float c[3] = {q.x, q.y, q.z};
    const int ci[3] = {cx0 >> L, cy0 >> L, cz0 >> L};
    if (counter < k) {
        const float st = __fsqrt_rn(np.thres);
        bool more = false;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            more |= (ci[d] - o >= 0) && st > fs_face_lo(c[d], np.a, (float)(ci[d] - o), h);
            more |= (ci[d] + o + 1 <= B) && st > fs_face_hi(c[d], np.a, (float)(ci[d] + o + 1), h);
        }
        return more;
    }
    const float r = __fsqrt_rn(kth);
    bool more = false;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        more |= (ci[d] - o >= 0) && r >= fs_face_lo(c[d], np.a, (float)(ci[d] - o), h);
        more |= (ci[d] + o + 1 <= B) && r >= fs_face_hi(c[d], np.a, (float)(ci[d] + o + 1), h);
    }
    return more;
}

// Batches admitting at least kMergeMin candidates are merged in one step:
// for lists of up to 64 slots by ranks (merge_rank) below kSortMin
// candidates, otherwise by a sorting network (merge_batch).  The rank merge's
// binary search and per-candidate loop grow with the list, and on lists of
// 65-96 slots the sorting network is faster throughout (measured on the
// 20M-point k=64 sheets).
#ifndef EGT_KNN_MERGE_MIN
#define EGT_KNN_MERGE_MIN 3
#endif
#ifndef EGT_KNN_SORT_MIN
#define EGT_KNN_SORT_MIN 24
#endif
constexpr int kMergeMin = EGT_KNN_MERGE_MIN;
constexpr int kSortMin = EGT_KNN_SORT_MIN;

// Offers one batch of candidates (one per lane, `adm` = admitted: d <= thres
// and d < the list's last slot) to the list.
//   kExact: the reference's appendDistanceGrid rule, one candidate at a time
//           in lane order (dedup, FindPosition on equal distances);
//   else:   sorted insertion, or one merge step for larger batches.  The two
//           agree whenever the kept distances are pairwise distinct; callers
//           discard results with equal distances (has_ties).
template <bool kExact, int S>
__device__ __forceinline__ void offer(WarpList<S>& L, float d, int p, bool adm, int lane, float* s_md, int* s_mp) {
    unsigned mask = __ballot_sync(0xffffffffu, adm);
    const int nb = __popc(mask);
    if (!kExact && nb >= kMergeMin) {
        if (S > 2 || nb >= kSortMin) merge_batch(L, d, p, adm, lane, s_md, s_mp);
        else merge_rank(L, d, p, adm, mask, lane, s_md, s_mp);
        return;
    }
    while (mask) {
        const int src = __ffs(mask) - 1;
        mask &= mask - 1;
        const float dd = __shfl_sync(0xffffffffu, d, src);
        const int pp = __shfl_sync(0xffffffffu, p, src);
        if (kExact) L.insert(dd, pp, lane);
        else insert_sorted(L, dd, pp, lane);
    }
}

// True when two of the first `keep` slots hold equal distances.
template <int S>
__device__ __forceinline__ bool has_ties(const WarpList<S>& L, int keep, int lane) {
    bool bad = false;
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        const float up = __shfl_up_sync(0xffffffffu, L.dist[s], 1);
        const float wrap = __shfl_sync(0xffffffffu, s > 0 ? L.dist[s > 0 ? s - 1 : 0] : 0.f, 31);
        const float prev = lane == 0 ? wrap : up;
        if (t >= 1 && t < keep && !(prev < L.dist[s])) bad = true;
    }
    return __any_sync(0xffffffffu, bad);
}

// A flattened candidate sequence over up to 32 point ranges (cells, or row
// ranges of cells).  After compaction the r-th non-empty range is held by
// lane r: sequence positions [incl of lane r-1, incl of lane r) map to
// order[cs + ...].  Lanes >= m hold incl = INT_MAX.
struct RangeSeq {
    int incl, cs, m, total;
};

// Builds the sequence from one range per lane (sz points starting at cs; sz
// = 0 for none).  s_pref / s_start: 32-int scratch of the calling warp.
__device__ __forceinline__ RangeSeq range_seq(int sz, int cs, int lane, int* s_pref, int* s_start) {
    int incl = sz;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const unsigned ne = __ballot_sync(0xffffffffu, sz > 0);
    RangeSeq q;
    q.total = __shfl_sync(0xffffffffu, incl, 31);
    q.m = __popc(ne);
    __syncwarp();
    if (sz > 0) {
        const int r = __popc(ne & ((1u << lane) - 1u));
        s_pref[r] = incl;
        s_start[r] = cs;
    }
    __syncwarp();
    q.incl = lane < q.m ? s_pref[lane] : INT_MAX;
    q.cs = lane < q.m ? s_start[lane] : 0;
    __syncwarp();  // the scratch may be rewritten by the next sequence
    return q;
}

// Point index of candidate base + lane of the sequence (-1 past its end).
// The range of every lane of the chunk comes from two warp votes: the number
// of ranges ending at or before `base`, and a mask of the positions inside
// the chunk where a new range starts.  `order` maps level order to sorted
// index (nullptr: identity).
__device__ __forceinline__ int seq_index(const RangeSeq& q, int base, int lane, const int* __restrict__ order) {
    const int before = __popc(__ballot_sync(0xffffffffu, q.incl <= base));
    const int at = q.incl - base;
    const unsigned starts = __reduce_or_sync(0xffffffffu, (at > 0 && at < 32) ? (1u << at) : 0u);
    const int c = before + __popc(starts & ((2u << lane) - 1u));
    const int prev_end = __shfl_sync(0xffffffffu, q.incl, (c - 1) & 31);
    const int cs = __shfl_sync(0xffffffffu, q.cs, c & 31);
    const int j = base + lane;
    if (j >= q.total) return -1;
    const int pos = cs + (j - (c > 0 ? prev_end : 0));
    return order ? __ldg(order + pos) : pos;
}

// Position of candidate point p (a dummy for no candidate or the query itself).
__device__ __forceinline__ float4 stream_point(int p, int q, const float4* __restrict__ p4) {
    return (p >= 0 && p != q) ? __ldg(p4 + p) : make_float4(0.f, 0.f, 0.f, 0.f);
}

// True when no point of the level-L cells x0..x1 of row (cy, cz) can be
// admitted to the list: the query's distance to their box, less a margin,
// squared, exceeds the admission threshold kth (admission needs d < kth).
// Float arithmetic with margins that cover its own rounding: the box bounds
// are off by ~1e-7 (normalised units), a point may sit ~1e-7 outside its
// cell's box (the float rounding of its cell key), and the float squared
// distances carry a relative error below 1e-6; the 2e-6 margin per axis and
// the 1e-5 relative margin on kth exceed all three, so a skipped row holds no
// admissible point.  Oversized cells are checked by the caller whatever their
// distance.
__device__ __forceinline__ bool cells_beyond(const NormParams& np, float4 pq, int lvl, int x0, int x1, int cy, int cz,
                                             float kth) {
    if (!(kth < 1e9f)) return false;  // list not full yet: everything is admitted
    const float h = __fmul_rn(__fsub_rn(np.b, np.a), (float)(1 << lvl) * (1.0f / 1024.0f));
    const float c[3] = {pq.x, pq.y, pq.z};
    const int c0[3] = {x0, cy, cz}, c1[3] = {x1 + 1, cy + 1, cz + 1};
    float d2 = 0.0f;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const float lo = np.a + (float)c0[d] * h, hi = np.a + (float)c1[d] * h;
        const float g = fmaxf(fmaxf(lo - c[d], c[d] - hi) - 2e-6f, 0.0f);
        d2 = fmaf(g, g, d2);
    }
    return d2 > kth * (1.0f + 1e-5f);
}

// Streams the points of `m` cells (cell l held by lane l as [cs, ce), ce < 0 =
// empty) through the list, in cell order.  Sets `invalid` when a visited cell
// holds >= max_pts points (GridKNNCuda.cu:672, 685): the cells before it are
// still processed, the rest are not.  skipL >= 0: skip points whose level-skipL
// cell lies in the 3x3x3 block around the query's level-skipL cell (qx, qy,
// qz), which the previous levels visited.
template <bool kExact, int S>
__device__ __forceinline__ void stream_cells(WarpList<S>& L, bool& invalid, int m, int cs, int ce,
                                             const int* __restrict__ order, const float4* __restrict__ p4,
                                             int q, float4 pq, float thres, int max_pts, int lane,
                                             int skipL, int qx, int qy, int qz, int* s_pref, int* s_start, float* s_md,
                                             int* s_mp, bool culled = false) {
    const bool exists = lane < m && ce >= 0;
    const bool big = exists && (ce - cs) >= max_pts;
    const unsigned bigmask = __ballot_sync(0xffffffffu, big);
    const int mlim = bigmask ? (__ffs(bigmask) - 1) : m;
    const int sz = (lane < mlim && exists && !culled) ? ce - cs : 0;
    const RangeSeq seq = range_seq(sz, cs, lane, s_pref, s_start);
    // Software pipeline over 32-candidate chunks: while chunk c is filtered
    // and offered, the position of chunk c+1 and the point index of chunk c+2
    // are in flight, so the dependent index -> position loads of a chunk never
    // wait in line.
    int pA = seq_index(seq, 32, lane, order);
    int pB = seq_index(seq, 0, lane, order);
    float4 vB = stream_point(pB, q, p4);
    for (int base = 0; base < seq.total; base += 32) {
        const int p = pB;
        const float4 v = vB;
        pB = pA;
        vB = stream_point(pB, q, p4);
        pA = seq_index(seq, base + 64, lane, order);
        float d = 1e30f;
        bool ok = false;
        if (p >= 0 && p != q) {
            bool fresh = true;
            if (skipL >= 0) {
                const uint32_t c = __float_as_uint(v.w);
                const int px = (int)((c & 1023u) >> skipL), py = (int)(((c >> 10) & 1023u) >> skipL),
                          pz = (int)(((c >> 20) & 1023u) >> skipL);
                fresh = abs(px - qx) > 1 || abs(py - qy) > 1 || abs(pz - qz) > 1;
            }
            if (fresh) {
                d = fs_dist3(pq.x, pq.y, pq.z, v.x, v.y, v.z);
                ok = d <= thres;
                ++L.ev;
            }
        }
        offer<kExact, S>(L, d, p, ok && d < L.kth, lane, s_md, s_mp);
    }
    if (bigmask) invalid = true;
}

// The whole reference search for query q.  Returns the level reached
// (kMaxLevels when the query ran out of levels).  kExact keeps the k-slot
// list of the reference's insertion rule; otherwise the list keeps k+1 slots
// (one more than the output) so that has_ties can check the k-th/(k+1)-th
// boundary.  Either way the decisions see the k-th smallest distance offered
// so far, which does not depend on the insertion rule.
template <bool kExact, int S>
__device__ int search(const KnnArgs& a, const NormParams& np, int q, float4 pq, WarpList<S>& L,
                      bool& invalid, int lane, int* s_pref, int* s_start, float* s_md, int* s_mp) {
    const uint32_t c0 = __float_as_uint(pq.w);
    const int cx0 = c0 & 1023, cy0 = (c0 >> 10) & 1023, cz0 = (c0 >> 20) & 1023;
    const int k = a.k;
    L.init(kExact ? k : k + 1);
    invalid = false;
    // offset 0 at level 0: the query's own cell (always occupied)
    int2 own = lane == 0 ? find_cell(a.lv[0], cx0, cy0, cz0) : make_int2(-1, -1);
    stream_cells<kExact, S>(L, invalid, 1, own.x, own.y, nullptr, a.p4, q, pq, np.thres, a.max_pts, lane, -1, 0, 0, 0,
                            s_pref, s_start, s_md, s_mp);
    bool cont = decide(np, 0, 0, L.counter, k, kExact ? L.kth : L.fetch_dist(k - 1), invalid, pq, cx0, cy0, cz0);
    int reached = 0;
    for (int lvl = 0; cont; lvl++) {
        reached = lvl;
        const LevelDev& LV = a.lv[lvl];
        int2 cell = make_int2(-1, -1);
        bool culled = false;
        if (lane < 26) {
            const int cx = (cx0 >> lvl) + kShell[lane][0], cy = (cy0 >> lvl) + kShell[lane][1],
                      cz = (cz0 >> lvl) + kShell[lane][2];
            cell = find_cell(LV, cx, cy, cz);
            culled = cell.x >= 0 && cells_beyond(np, pq, lvl, cx, cx, cy, cz, L.kth);
        }
        const int sL = max(lvl - 1, 0);
        stream_cells<kExact, S>(L, invalid, 26, cell.x, cell.y, LV.order, a.p4, q, pq, np.thres, a.max_pts, lane,
                                lvl - 1, cx0 >> sL, cy0 >> sL, cz0 >> sL, s_pref, s_start, s_md, s_mp, culled);
        cont = decide(np, lvl, 1, L.counter, k, kExact ? L.kth : L.fetch_dist(k - 1), invalid, pq, cx0, cy0, cz0);
        if (lvl == kMaxLevels - 1) break;
    }
    // still searching after the B = 8 ring: invalid (GridKNNCuda.cu:2572-2586)
    if (cont) { invalid = true; reached = kMaxLevels; }
    return reached;
}

// One query of the plain search: the fast list rule first; if the k+1 kept
// distances are not pairwise distinct the order of equal distances matters
// and the query is searched again with the reference's exact rule.
template <bool kFast, int S>
__device__ __forceinline__ int plain_query(const KnnArgs& a, const NormParams& np, int q, float4 pq, WarpList<S>& L,
                                           bool& invalid, int lane, int* s_pref, int* s_start, float* s_md,
                                           int* s_mp, bool& rerun) {
    rerun = false;
    if (kFast) {
        const int reached = search<false, S>(a, np, q, pq, L, invalid, lane, s_pref, s_start, s_md, s_mp);
        if (!has_ties(L, min(L.counter, a.k + 1), lane)) return reached;
        rerun = true;
    }
    return search<true, S>(a, np, q, pq, L, invalid, lane, s_pref, s_start, s_md, s_mp);
}

// Writes the outputs of query q from its final list.
template <int S>
__device__ __forceinline__ void write_query(const KnnArgs& a, int q, const WarpList<S>& L, bool invalid, int reached,
                                            int lane) {
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        if (t < a.k) a.lists[(size_t)q * a.k + t] = invalid ? -1 : L.idx[s];
    }
    const float kth = L.fetch_dist(a.k - 1);
    if (lane == 0) {
        if (a.kth_out) a.kth_out[q] = (!invalid && L.counter >= a.k) ? kth : 1e10f;
        if (a.qlevel) a.qlevel[q] = (uint8_t)reached;
        if (invalid) atomicAdd(&a.counters[kCtrInvalid], 1ull);
        atomicMax(&a.counters[kCtrMaxLevel], (unsigned long long)reached);
    }
}

// Default number of queries a warp of the persistent kNN kernels claims per
// atomic (KnnArgs::chunk).
constexpr int kChunk = 4;

// Next chunk of queries for the calling warp (uniform); >= n when done.
__device__ __forceinline__ int claim(const KnnArgs& a, int lane, int n) {
    unsigned long long q0 = 0;
    if (lane == 0) q0 = atomicAdd(a.work ? a.work : &a.counters[kCtrWork], (unsigned long long)a.chunk);
    return (int)min(__shfl_sync(0xffffffffu, q0, 0), (unsigned long long)n);
}

}  // namespace
}  // namespace egt
