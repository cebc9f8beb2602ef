// Exact self-kNN over the cell hierarchy with the reference's semantics.
//
// Reference: GridStructure::GRIDCUDAKNNSELF_COMPACT (GridKNNCuda.cu:2322-2634)
// and its kernel construct_neighbors_self_compact (GridKNNCuda.cu:647-743).
// The reference runs one launch per shell cell (27 launches for the own cell
// and ring 1, 26 per further level), each followed by a device sync, a host
// reduction and a compaction of the still-searching queries.  Here one warp
// runs a query through the whole sequence in a single launch:
//
//   own level-0 cell; decide; ring 1 at level 0; decide; ring 1 at level 1; ...
//   ring 1 at level 7 (B = 8); a query still searching after that is invalid.
//
// The candidate order is the reference's: cells in its shell nest order, the
// points of a cell in ascending sorted index (the stable level sort), and the
// list is updated by the exact appendDistanceGrid rule (knn_common.cuh), so
// the produced lists -- including the order of equal distances -- are
// bit-identical to the reference's.  The 26 shell cells of a level are
// resolved in parallel (one per lane) and their points are streamed as one
// flattened candidate sequence, 32 candidates per step.
//
// Re-visits are skipped: the cells visited up to level L-1 form the 3x3x3
// block of level L-1 around the query, and the level-L ring covers it again.
// A point of that block was already offered to the list: it is either in the
// list (the dedup rule rejects it) or farther than the k-th distance of that
// time, which never grows (the admission rule rejects it), so offering it again
// cannot change the list.
#include <atomic>
#include <cub/cub.cuh>
#include <map>
#include <vector>
#include <mutex>

#include "egt_internal.cuh"
#include "knn_common.cuh"
#include "knn_search.cuh"
#include "knn_select.cuh"
#include "proposal.cuh"
#include "knn_tile.cuh"

namespace egt {
namespace {

// Persistent: one resident wave of blocks whose warps claim a.chunk queries at
// a time, so that a warp that drew cheap queries moves on instead of idling
// until the most expensive query of its block is done.
template <int S, bool kFast>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) k_knn_plain(KnnArgs a) {
    __shared__ int s_pref[kWarps][32];
    __shared__ int s_start[kWarps][32];
    __shared__ float s_md[kWarps][32 * S];
    __shared__ int s_mp[kWarps][32 * S];
    __shared__ unsigned s_rerun;
    if (threadIdx.x == 0) s_rerun = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const NormParams np = *a.np;
    unsigned evals = 0;  // candidate distances this lane evaluated
    const int n = launch_size(a);
    for (int q0 = claim(a, lane, n); q0 < n; q0 = claim(a, lane, n)) {
        const int q1 = min(q0 + a.chunk, n);
        for (int jq = q0; jq < q1; jq++) {
            const int q = a.qmap ? a.qmap[jq] : jq;
            const float4 pq = a.p4[q];
            WarpList<S> L;
            bool invalid, rerun;
            const int reached = plain_query<kFast, S>(a, np, q, pq, L, invalid, lane, s_pref[w], s_start[w], s_md[w],
                                                      s_mp[w], rerun);
            write_query<S>(a, q, L, invalid, reached, lane);
            if (rerun && lane == 0) atomicAdd(&s_rerun, 1u);
            evals += L.ev;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) evals += __shfl_xor_sync(0xffffffffu, evals, o);
    if (lane == 0 && evals) atomicAdd(&a.counters[kCtrEvals], (unsigned long long)evals);
    __syncthreads();
    if (threadIdx.x == 0 && s_rerun) atomicAdd(&a.counters[kCtrExactRerun], (unsigned long long)s_rerun);
}

// Block-selection search (knn_select.cuh), persistent like k_knn_plain.  A
// query it cannot certify runs the ring search right away in the same warp
// (plain_query; S = list registers per lane for k+1 slots), so the rare slow
// queries overlap with the rest of the launch.
template <int S>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) k_knn_select(KnnArgs a) {
    __shared__ SelScratch s_sc[kWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    SelScratch& sc = s_sc[w];
    const NormParams np = *a.np;
    // every distance admitted (the under-full rule then always continues)
    const bool usable = np.thres > 4.0f;
    const int n = launch_size(a);
    unsigned evals = 0, ring = 0, reruns = 0;
    int gstart = 0, maxlevel = 0;
    for (int q0 = claim(a, lane, n); q0 < n; q0 = claim(a, lane, n)) {
        const int q1 = min(q0 + a.chunk, n);
        for (int jq = q0; jq < q1; jq++) {
            const int q = a.qmap ? a.qmap[jq] : jq;
            const float4 pq = a.p4[q];
            SelOut r{false, 0, 0.0f};
            if (usable) r = sel_query(a, np, q, pq, lane, sc, gstart, evals);
            if (r.ok) {
                if (lane == 0) {
                    if (a.kth_out) a.kth_out[q] = r.kth;
                    if (a.qlevel) a.qlevel[q] = (uint8_t)r.reached;
                    maxlevel = max(maxlevel, r.reached);
                }
                continue;
            }
            WarpList<S> L;
            bool invalid, rerun;
            const int reached = plain_query<true, S>(a, np, q, pq, L, invalid, lane, sc.pref, sc.start, sc.cd, sc.cj,
                                                     rerun);
            write_query<S>(a, q, L, invalid, reached, lane);
            __syncwarp();  // the scratch is rewritten by the next query
            evals += L.ev;
            ++ring;
            reruns += rerun ? 1u : 0u;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) evals += __shfl_xor_sync(0xffffffffu, evals, o);
    if (lane == 0) {
        if (evals) atomicAdd(&a.counters[kCtrEvals], (unsigned long long)evals);
        if (maxlevel) atomicMax(&a.counters[kCtrMaxLevel], (unsigned long long)maxlevel);
        if (ring) atomicAdd(a.n_ring ? a.n_ring : &a.counters[kCtrSelFallback], (unsigned long long)ring);
        if (reruns) atomicAdd(&a.counters[kCtrExactRerun], (unsigned long long)reruns);
    }
}

// ---------------------------------------------------------------------------
// Proposal-driven search (an extension of this project).  The query's box
// (class from the proposal network) is searched for its k+1 smallest
// distances.  The result is accepted only when it provably equals the plain
// search's list:
//   (1) >= k candidates and the k+1 smallest distances pairwise distinct, so
//       the sorted list does not depend on the candidate order;
//   (2) the ball of radius sqrt(kth) + margin lies inside the searched box,
//       so no point outside it is as near as the k-th: the k kept points are
//       the k nearest of the cloud, G;
//   (3) the plain search's stop step sf is replayed with decide(): once the
//       plain search's visited block contains G its list is G and it stops
//       exactly where decide(kth(G)) says so; before that its k-th distance is
//       >= kth(G) (or its list is under-full) and it continues whenever
//       decide(kth(G)) and the under-full branch both continue.  Every point
//       of G must be visited by step sf;
//   (4) no cell of the levels visited up to sf holds >= max_points_in_cell
//       points (the plain search would have invalidated the query).
// The box's candidates below its cut are collected and the k+1 smallest
// selected once (select_list).  A failed check, or a box whose candidates do
// not fit the collection buffer, runs the plain search for the query.

// Streams the points of m row ranges (range l held by lane l as [cs, ce)),
// software-pipelined as in stream_cells, through the list, admitting only
// distances below `cut` as well.
template <int S>
__device__ __forceinline__ void stream_ranges(WarpList<S>& L, int m, int cs, int ce, const int* __restrict__ order,
                                              const float4* __restrict__ p4, int q, float4 pq, float thres, float cut,
                                              int lane, int* s_pref, int* s_start, float* s_md, int* s_mp) {
    const RangeSeq seq = range_seq(lane < m ? ce - cs : 0, cs, lane, s_pref, s_start);
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
            d = fs_dist3(pq.x, pq.y, pq.z, v.x, v.y, v.z);
            ok = d <= thres;
        }
        offer<false, S>(L, d, p, ok && d < L.kth && d < cut, lane, s_md, s_mp);
    }
}

// For lists of more than 64 slots the box candidates are not merged into the
// list as they stream: every candidate below the box's cut is collected into
// a per-warp buffer, and the k+1 smallest are selected once at the end
// (select_list).  Merging costs grow with the list; selection costs do not
// (measured on the 20M-point k=64 sheets: 153 ms merged, 107 ms collected;
// on the 4M-point k=40 superquadrics merging stays ahead, 19.4 ms against
// 20.6 ms).  Per-warp scratch of the proposal-driven kernel, in dynamic
// shared memory.
constexpr int kCollectCap = 448;  // candidates collected per box (more: the query runs the plain search)
constexpr int kSelectCap = 128;   // selected candidates plus the boundary bucket
constexpr int kBuckets = 256;
struct BoxScratch {
    float* cd;   // [kCollectCap] collected distances
    int* cp;     // [kCollectCap] collected points
    int* hist;   // [kBuckets]
    float* sd;   // [kSelectCap] selected candidates in bucket order
    int* sp;
};
constexpr size_t kBoxScratchBytes = (size_t)kCollectCap * 8 + kBuckets * 4 + kSelectCap * 8;

__device__ __forceinline__ BoxScratch box_scratch(unsigned char* base, int warp) {
    unsigned char* w = base + (size_t)warp * kBoxScratchBytes;
    BoxScratch b;
    b.cd = reinterpret_cast<float*>(w);
    b.cp = reinterpret_cast<int*>(w + kCollectCap * 4);
    b.hist = reinterpret_cast<int*>(w + kCollectCap * 8);
    b.sd = reinterpret_cast<float*>(w + kCollectCap * 8 + kBuckets * 4);
    b.sp = reinterpret_cast<int*>(w + kCollectCap * 8 + kBuckets * 4 + kSelectCap * 4);
    return b;
}

// Streams the points of m row ranges (range l held by lane l as [cs, ce)),
// software-pipelined as in stream_cells, collecting every candidate with
// d <= thres and d < cut.  Returns the new collected count
// (uniform; it may exceed kCollectCap, in which case the excess is dropped and
// the caller gives up).  dmax: the lane's largest collected distance.
__device__ __forceinline__ int stream_collect(int m, int cs, int ce, const int* __restrict__ order,
                                              const float4* __restrict__ p4, int q, float4 pq, float thres, float cut,
                                              int lane, int* s_pref, int* s_start, const BoxScratch& bx, int count,
                                              float& dmax) {
    const RangeSeq seq = range_seq(lane < m ? ce - cs : 0, cs, lane, s_pref, s_start);
    int pA = seq_index(seq, 32, lane, order);
    int pB = seq_index(seq, 0, lane, order);
    float4 vB = stream_point(pB, q, p4);
    for (int base = 0; base < seq.total; base += 32) {
        const int p = pB;
        const float4 v = vB;
        pB = pA;
        vB = stream_point(pB, q, p4);
        pA = seq_index(seq, base + 64, lane, order);
        float d = 0.0f;
        bool ok = false;
        if (p >= 0 && p != q) {
            d = fs_dist3(pq.x, pq.y, pq.z, v.x, v.y, v.z);
            ok = d <= thres && d < cut;
        }
        const unsigned mk = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            const int at = count + __popc(mk & ((1u << lane) - 1u));
            if (at < kCollectCap) { bx.cd[at] = d; bx.cp[at] = p; }
            dmax = fmaxf(dmax, d);
        }
        count += __popc(mk);
    }
    return count;
}

// (r - margin)^2 rounded down, r = the query's distance to the nearest
// in-grid face of the box sub-box of y/z half-width `ring` (0 when r <= margin;
// 3e38 when no face is inside the grid).  A squared distance below it gives a
// ball that passes ball_in_box for that sub-box.
__device__ __forceinline__ float ring_inner_sq(const NormParams& np, float4 pq, int cls, int ring, uint32_t c0) {
    int lo[3], end[3];
    box_bounds(cls, ring, c0, lo, end);
    const double h0 = (double)__fmul_rn(__fsub_rn(np.b, np.a), 1.0f / 1024.0f);
    const double c[3] = {pq.x, pq.y, pq.z};
    double fnear = 1e30;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        if (lo[d] > 0) fnear = fmin(fnear, c[d] - ((double)np.a + lo[d] * h0));
        if (end[d] < 1024) fnear = fmin(fnear, ((double)np.a + end[d] * h0) - c[d]);
    }
    if (fnear >= 1e29) return 3.0e38f;
    const double t = fnear - kBoxMargin;
    return t > 0.0 ? __double2float_rd(t * t) : 0.0f;
}

// Bucket of a collected distance: 256 buckets, linear in d over [0, dmax]
// (monotone in d, so bucket order never contradicts distance order).
__device__ __forceinline__ int dist_bucket(float d, float scale) {
    return min((int)__fmul_rn(d, scale), kBuckets - 1);
}

// Puts the `need` smallest of the `count` collected candidates, ordered by
// (distance, index), into slots [0, need) of L (need <= L.k).  A counting
// pass over 256 distance buckets finds the bucket holding the need-th
// smallest; the candidates of that and lower buckets are placed in bucket
// order and ranked inside their bucket.  Returns false when those candidates
// do not fit in the selection buffer.
template <int S>
__device__ bool select_list(WarpList<S>& L, const BoxScratch& bx, int count, int need, float dmax, float* md,
                            int* mp, int lane) {
    const float scale = dmax > 0.0f ? __fdiv_rn(255.99f, dmax) : 0.0f;
#pragma unroll
    for (int i = 0; i < kBuckets / 32; i++) bx.hist[lane + 32 * i] = 0;
    __syncwarp();
    for (int e = lane; e < count; e += 32) atomicAdd(&bx.hist[dist_bucket(bx.cd[e], scale)], 1);
    __syncwarp();
    // lane l owns buckets [8l, 8l+8)
    int c8[kBuckets / 32], sum = 0;
#pragma unroll
    for (int i = 0; i < kBuckets / 32; i++) { c8[i] = bx.hist[lane * (kBuckets / 32) + i]; sum += c8[i]; }
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int excl = incl - sum;
    const int target = need - 1;  // rank of the last selected candidate
    const int wl = __ffs(__ballot_sync(0xffffffffu, excl <= target && target < incl)) - 1;
    int bstar = 0, below = 0;
    if (lane == wl) {
        int acc = excl;
#pragma unroll
        for (int i = 0; i < kBuckets / 32; i++) {
            if (acc + c8[i] > target) { bstar = lane * (kBuckets / 32) + i; below = acc; break; }
            acc += c8[i];
        }
    }
    bstar = __shfl_sync(0xffffffffu, bstar, wl);
    below = __shfl_sync(0xffffffffu, below, wl);
    const int tot = below + bx.hist[bstar];
    __syncwarp();
    if (tot > kSelectCap) return false;
    // bucket starts (exclusive prefix) for the buckets that take part
    {
        int run = excl;
#pragma unroll
        for (int i = 0; i < kBuckets / 32; i++) {
            const int b = lane * (kBuckets / 32) + i;
            if (b <= bstar) bx.hist[b] = run;
            run += c8[i];
        }
    }
    __syncwarp();
    for (int e = lane; e < count; e += 32) {
        const float d = bx.cd[e];
        const int b = dist_bucket(d, scale);
        if (b <= bstar) {
            const int slot = atomicAdd(&bx.hist[b], 1);
            bx.sd[slot] = d;
            bx.sp[slot] = bx.cp[e];
        }
    }
    __syncwarp();
    // hist[b] is now the end of bucket b, and the start of bucket b+1
    for (int i = lane; i < tot; i += 32) {
        const float d = bx.sd[i];
        const int p = bx.sp[i];
        const int b = dist_bucket(d, scale);
        int r = b > 0 ? bx.hist[b - 1] : 0;
        const int e1 = bx.hist[b];
        for (int j = r; j < e1; j++) {
            const float dj = bx.sd[j];
            r += (dj < d || (dj == d && bx.sp[j] < p)) ? 1 : 0;
        }
        if (r < need) { md[r] = d; mp[r] = p; }
    }
    __syncwarp();
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        L.dist[s] = t < need ? md[t] : 1e10f;
        L.idx[s] = t < need ? mp[t] : -1;
    }
    __syncwarp();
    L.counter = need;
    L.kth = L.fetch_dist(L.k - 1);
    return true;
}

// Box search + certification.  Returns true with L holding the plain
// search's list in slots [0, k) and `reached` its level.
template <int S>
__device__ bool box_search(const KnnArgs& a, const NormParams& np, int q, float4 pq, int cls, WarpList<S>& L,
                           int lane, int* s_pref, int* s_start, float* s_md, int* s_mp, const BoxScratch& bx,
                           int& reached) {
    const int lvl = kBoxClass[cls][0], R = kBoxClass[cls][1];
    const LevelDev& LV = a.lv[lvl];
    const uint32_t c0 = __float_as_uint(pq.w);
    const int cx0 = c0 & 1023u, cy0 = (c0 >> 10) & 1023u, cz0 = (c0 >> 20) & 1023u;
    const int cix = cx0 >> lvl, ciy = cy0 >> lvl, ciz = cz0 >> lvl;
    const int k = a.k;
    L.init(k + 1);
    // A certified result has sqrt(kth) + margin below every in-grid face
    // distance of the box, so distances at or above the nearest face distance,
    // squared, can neither enter G nor tie with its k-th: they are not admitted.
    float cut = 3.0e38f;
    {
        int lo[3], end[3];
        box_bounds(cls, R, c0, lo, end);
        const double h0 = (double)__fmul_rn(__fsub_rn(np.b, np.a), 1.0f / 1024.0f);
        const double c[3] = {pq.x, pq.y, pq.z};
        double fnear = 1e30;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (lo[d] > 0) fnear = fmin(fnear, c[d] - ((double)np.a + lo[d] * h0));
            if (end[d] < 1024) fnear = fmin(fnear, ((double)np.a + end[d] * h0) - c[d]);
        }
        if (fnear < 1e29) cut = __double2float_ru(fmax(fnear, 0.0) * fmax(fnear, 0.0));
    }
    const int nrows = (2 * R + 1) * (2 * R + 1);
    constexpr bool kCollect = S > 2;
    int count = 0, ring = -1;
    float dmax = 0.0f;
    bool enough = false;
    // Rows are streamed 32 per round, ring by ring.  After a round that
    // completes a ring: once k candidate distances lie
    // below its sub-box's inner radius (less the margin), squared, the k
    // nearest points of the cloud -- and every point as near as the k-th --
    // have been streamed, and the rest of the box cannot change the list up
    // to its k-th slot or the tie check there.
    for (int rb = 0; rb < nrows && !enough;) {
        const int re = min(rb + 32, nrows);
        int2 rg = make_int2(0, 0);
        const int t = rb + lane;
        if (t < re) {
            // merged lists skip rows whose points all lie beyond the admission
            // bound (measured: a gain there, a loss for the collecting path)
            const int ry = ciy + kRowOrder[t][0], rz = ciz + kRowOrder[t][1];
            if (kCollect || !cells_beyond(np, pq, lvl, cix - R, cix + R, ry, rz, fminf(cut, L.kth)))
                rg = row_points(LV, cix - R, cix + R, ry, rz);
        }
        const int* order = lvl ? LV.order : nullptr;
        if constexpr (kCollect) {
            count = stream_collect(re - rb, rg.x, rg.y, order, a.p4, q, pq, np.thres, cut, lane, s_pref, s_start,
                                   bx, count, dmax);
            if (count > kCollectCap) return false;
        } else {
            stream_ranges<S>(L, re - rb, rg.x, rg.y, order, a.p4, q, pq, np.thres, cut, lane, s_pref, s_start, s_md,
                             s_mp);
        }
        rb = re;
        int j = ring;
        while ((2 * j + 3) * (2 * j + 3) <= rb) j++;
        if (j > ring) {
            ring = j;
            if (ring < R) {
                const float inner = ring_inner_sq(np, pq, cls, ring, c0);
                if constexpr (kCollect) {
                    if (count >= k) {
                        int below = 0;
                        for (int e = lane; e < count; e += 32) below += bx.cd[e] < inner ? 1 : 0;
                        enough = __reduce_add_sync(0xffffffffu, below) >= k;
                    }
                } else {
                    enough = L.counter >= k && L.fetch_dist(k - 1) < inner;
                }
            }
        }
    }
    if constexpr (kCollect) {
        if (count < k) return false;
        dmax = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(dmax)));  // d >= 0: bit order
        if (!select_list<S>(L, bx, count, min(count, k + 1), dmax, s_md, s_mp, lane)) return false;
    } else if (L.counter < k) {
        return false;
    }
    // (2) the k-th ball lies inside the searched box (the sub-box of `ring`
    // when the search stopped early)
    {
        int lo[3], end[3];
        box_bounds(cls, enough ? ring : R, c0, lo, end);
        if (!ball_in_box(np, pq, L.fetch_dist(k - 1), lo, end)) return false;
    }
    // (1) the kept distances are strictly increasing
    if (has_ties(L, min(L.counter, k + 1), lane)) return false;
    const float kth = L.fetch_dist(k - 1);
    // (3) the plain stop step sf.  When thres exceeds every face distance of
    // the unit cube (sqrt(thres) > 2) the under-full branch continues wherever
    // the full branch does, and need not be evaluated.
    const bool huge = np.thres > 4.0f;
    int sf = -1;
    for (int st = 0; st <= kMaxLevels; st++) {
        const int Ls = st == 0 ? 0 : st - 1, o = st == 0 ? 0 : 1;
        if (!decide(np, Ls, o, k, k, kth, false, pq, cx0, cy0, cz0)) { sf = st; break; }
        if (!huge && !decide(np, Ls, o, 0, k, kth, false, pq, cx0, cy0, cz0)) return false;
    }
    if (sf < 0) return false;
    // G lies in the block visited by step sf: at once when the k-th ball
    // (with the margin) does, else point by point.
    {
        const int Lf = sf == 0 ? 0 : sf - 1, of = sf == 0 ? 0 : 1;
        const int ci[3] = {cx0 >> Lf, cy0 >> Lf, cz0 >> Lf};
        int lo[3], end[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            lo[d] = (ci[d] - of) << Lf;
            end[d] = (ci[d] + of + 1) << Lf;
        }
        if (!ball_in_box(np, pq, kth, lo, end)) {
            int sg = 0;
#pragma unroll
            for (int s = 0; s < S; s++) {
                const int t = lane + 32 * s;
                if (t < k) sg = max(sg, visit_step(__float_as_uint(a.p4[L.idx[s]].w), c0));
            }
            if (__reduce_max_sync(0xffffffffu, sg) > sf) return false;
        }
    }
    // (4) no oversized cell on the visited levels
    for (int l = 0; l <= max(sf - 1, 0); l++)
        if (a.counters[kCtrMaxPop + l] >= (unsigned long long)a.max_pts) return false;
    reached = max(sf - 1, 0);
    return true;
}

template <int S>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) k_knn_learned(KnnArgs a, const uint8_t* __restrict__ cls) {
    extern __shared__ __align__(16) unsigned char s_scratch[];  // kWarps * kBoxScratchBytes
    __shared__ int s_pref[kWarps][32];
    __shared__ int s_start[kWarps][32];
    __shared__ float s_md[kWarps][32 * S];
    __shared__ int s_mp[kWarps][32 * S];
    __shared__ unsigned s_box, s_cert, s_rerun;
    if (threadIdx.x == 0) { s_box = 0; s_cert = 0; s_rerun = 0; }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const NormParams np = *a.np;
    const int n = launch_size(a);
    for (int q0 = claim(a, lane, n); q0 < n; q0 = claim(a, lane, n)) {
        const int q1 = min(q0 + a.chunk, n);
        for (int jq = q0; jq < q1; jq++) {
            const int q = a.qmap ? a.qmap[jq] : jq;
            const float4 pq = a.p4[q];
            WarpList<S> L;
            bool invalid = false, ok = false;
            int reached = 0;
            const int c = cls[q];
            if (c < kPropPlain) {
                ok = box_search<S>(a, np, q, pq, c, L, lane, s_pref[w], s_start[w], s_md[w], s_mp[w],
                                   box_scratch(s_scratch, w), reached);
                if (lane == 0) {
                    atomicAdd(&s_box, 1u);
                    if (ok) atomicAdd(&s_cert, 1u);
                }
            }
            if (!ok) {
                bool rerun;
                reached = plain_query<true, S>(a, np, q, pq, L, invalid, lane, s_pref[w], s_start[w], s_md[w],
                                               s_mp[w], rerun);
                if (rerun && lane == 0) atomicAdd(&s_rerun, 1u);
            }
            write_query<S>(a, q, L, invalid, reached, lane);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_box) {
        atomicAdd(&a.counters[kCtrBoxTried], (unsigned long long)s_box);
        atomicAdd(&a.counters[kCtrCertified], (unsigned long long)s_cert);
    }
    if (threadIdx.x == 0 && s_rerun) atomicAdd(&a.counters[kCtrExactRerun], (unsigned long long)s_rerun);
}

// ---------------------------------------------------------------------------
// Query-vs-reference kNN: GridStructure::GRIDCUDAKNNCompact (GridKNNCuda.cu:
// 1645-1939) with its kernel construct_neighbors (GridKNNCuda.cu:340-438) and
// GetKNNIndexes (:1941-1968).  The schedule is the self search's (own level-0
// cell, then the 26-cell shell at levels 0..7, invalid when still searching
// after B = 8), with the reference's differences for foreign queries:
//   * a query is normalised with the reference cloud's cube and may lie
//     outside it; its cell at level L is (int)(u * B_L), u = (x - a)/(b - a)
//     (:349-351), truncated toward zero, so it is computed per level rather
//     than shifted from level 0;
//   * no point is excluded as "self", and admission is d < thres (:357-363);
//   * with fewer than k neighbours the search continues when sqrt(thres) >=
//     a face distance (:377-392; the self search uses >);
//   * cells outside the grid are skipped without invalidating (:352-354).
__device__ __forceinline__ bool decide_query(const NormParams& np, int L, int o, int counter, int k, float kth,
                                             bool invalid, float4 q, const int ci[3]) {
    if (invalid) return false;
    const int B = 1024 >> L;
    const float h = __fdiv_rn(__fsub_rn(np.b, np.a), (float)B);
    const float c[3] = {q.x, q.y, q.z};
    const float r = counter < k ? __fsqrt_rn(np.thres) : __fsqrt_rn(kth);
    bool more = false;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        more |= (ci[d] - o >= 0) && r >= fs_face_lo(c[d], np.a, (float)(ci[d] - o), h);
        more |= (ci[d] + o + 1 <= B) && r >= fs_face_hi(c[d], np.a, (float)(ci[d] + o + 1), h);
    }
    return more;
}

template <bool kExact, int S>
__device__ int search_query(const KnnArgs& a, const NormParams& np, float4 pq, const float u[3], float thres_lt,
                            WarpList<S>& L, bool& invalid, int lane, int* s_pref, int* s_start, float* s_md,
                            int* s_mp) {
    const int k = a.k;
    L.init(kExact ? k : k + 1);
    invalid = false;
    int ci[3], cp[3];
#pragma unroll
    for (int d = 0; d < 3; d++) ci[d] = (int)__fmul_rn(u[d], 1024.0f);
    int2 own = lane == 0 ? find_cell(a.lv[0], ci[0], ci[1], ci[2]) : make_int2(-1, -1);
    stream_cells<kExact, S>(L, invalid, 1, own.x, own.y, nullptr, a.p4, -1, pq, thres_lt, a.max_pts, lane, -1, 0, 0,
                            0, s_pref, s_start, s_md, s_mp);
    bool cont = decide_query(np, 0, 0, L.counter, k, kExact ? L.kth : L.fetch_dist(k - 1), invalid, pq, ci);
    int reached = 0;
    for (int lvl = 0; cont; lvl++) {
        reached = lvl;
        const LevelDev& LV = a.lv[lvl];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            cp[d] = (int)__fmul_rn(u[d], (float)(1024 >> max(lvl - 1, 0)));  // the block visited so far
            ci[d] = (int)__fmul_rn(u[d], (float)(1024 >> lvl));
        }
        int2 cell = make_int2(-1, -1);
        bool culled = false;
        if (lane < 26) {
            const int cx = ci[0] + kShell[lane][0], cy = ci[1] + kShell[lane][1], cz = ci[2] + kShell[lane][2];
            cell = find_cell(LV, cx, cy, cz);
            culled = cell.x >= 0 && cells_beyond(np, pq, lvl, cx, cx, cy, cz, L.kth);
        }
        stream_cells<kExact, S>(L, invalid, 26, cell.x, cell.y, LV.order, a.p4, -1, pq, thres_lt, a.max_pts, lane,
                                lvl - 1, cp[0], cp[1], cp[2], s_pref, s_start, s_md, s_mp, culled);
        cont = decide_query(np, lvl, 1, L.counter, k, kExact ? L.kth : L.fetch_dist(k - 1), invalid, pq, ci);
        if (lvl == kMaxLevels - 1) break;
    }
    if (cont) { invalid = true; reached = kMaxLevels; }
    return reached;
}

// qpos: normalised query positions; query j (processing order a.qmap[j]) is
// row a.qmap[j] of out, in original reference ids (perm), -1 padded; an
// invalid query's row is all -1 (negateNotValidKnnIndexes, :291-302).
template <int S>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) k_knn_query(KnnArgs a, const float4* __restrict__ qpos,
                                                                     const int* __restrict__ perm,
                                                                     int* __restrict__ out) {
    __shared__ int s_pref[kWarps][32];
    __shared__ int s_start[kWarps][32];
    __shared__ float s_md[kWarps][32 * S];
    __shared__ int s_mp[kWarps][32 * S];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const NormParams np = *a.np;
    const float thres_lt = nextafterf(np.thres, 0.0f);  // d <= thres_lt  <=>  d < thres
    const float ab = __fsub_rn(np.b, np.a);
    const int n = launch_size(a);
    for (int q0 = claim(a, lane, n); q0 < n; q0 = claim(a, lane, n)) {
        const int q1 = min(q0 + a.chunk, n);
        for (int jq = q0; jq < q1; jq++) {
            const int row = a.qmap[jq];
            const float4 pq = qpos[row];
            const float u[3] = {__fdiv_rn(__fsub_rn(pq.x, np.a), ab), __fdiv_rn(__fsub_rn(pq.y, np.a), ab),
                                __fdiv_rn(__fsub_rn(pq.z, np.a), ab)};
            WarpList<S> L;
            bool invalid;
            search_query<false, S>(a, np, pq, u, thres_lt, L, invalid, lane, s_pref[w], s_start[w], s_md[w], s_mp[w]);
            if (has_ties(L, min(L.counter, a.k + 1), lane)) {
                search_query<true, S>(a, np, pq, u, thres_lt, L, invalid, lane, s_pref[w], s_start[w], s_md[w],
                                      s_mp[w]);
                if (lane == 0) atomicAdd(&a.counters[kCtrExactRerun], 1ull);
            }
#pragma unroll
            for (int s = 0; s < S; s++) {
                const int t = lane + 32 * s;
                if (t < a.k) {
                    const int v = L.idx[s];
                    out[(size_t)row * a.k + t] = (invalid || v < 0) ? -1 : perm[v];
                }
            }
            if (lane == 0 && invalid) atomicAdd(&a.counters[kCtrInvalid], 1ull);
        }
    }
}

// Normalised query positions (normalize_points, GridKNNCuda.cu:841-849, with
// the reference cloud's cube) and their level-0 cell keys for the processing
// order (cells outside the grid clamp to its border: order only).
__global__ void k_query_prepare(const float* __restrict__ xyz, int nq, const NormParams* __restrict__ np,
                                float4* __restrict__ qpos, uint32_t* __restrict__ key, int* __restrict__ idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const float mn = np->mn, d = __fsub_rn(np->mx, np->mn);
    float4 p;
    p.x = __fdiv_rn(__fsub_rn(xyz[3 * (size_t)i], mn), d);
    p.y = __fdiv_rn(__fsub_rn(xyz[3 * (size_t)i + 1], mn), d);
    p.z = __fdiv_rn(__fsub_rn(xyz[3 * (size_t)i + 2], mn), d);
    p.w = 0.0f;
    qpos[i] = p;
    const int cx = min(max(cell_coord(p.x, np->a, np->b, 1024), 0), 1023);
    const int cy = min(max(cell_coord(p.y, np->a, np->b, 1024), 0), 1023);
    const int cz = min(max(cell_coord(p.z, np->a, np->b, 1024), 0), 1023);
    key[i] = (uint32_t)cx | ((uint32_t)cy << 10) | ((uint32_t)cz << 20);
    idx[i] = i;
}

// Blocks of one resident wave of a persistent kernel, per (kernel, device).
template <typename K>
egt_status wave_blocks(K kernel, int64_t n, unsigned* out, size_t dyn_smem = 0) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> cache;
    int dev = 0;
    EGT_CUDA_TRY(cudaGetDevice(&dev));
    const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
    int blocks = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) blocks = it->second;
    }
    if (!blocks) {
        int sms = 0, per = 0;
        EGT_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        EGT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kWarps * 32, dyn_smem));
        blocks = std::max(1, sms * std::max(per, 1));
        std::lock_guard<std::mutex> lock(mu);
        cache[key] = blocks;
    }
    const int64_t need = (n + kWarps * kChunk - 1) / (kWarps * kChunk);  // enough for the default chunk
    *out = (unsigned)std::max<int64_t>(1, std::min<int64_t>(blocks, need));
    return EGT_OK;
}

template <int S>
egt_status launch_learned(const KnnArgs& a, const uint8_t* cls, cudaStream_t st) {
    constexpr size_t smem = S > 2 ? kWarps * kBoxScratchBytes : 0;  // collection buffers (box_search)
    static std::atomic<uint64_t> attr_set{0};  // per device
    int dev = 0;
    EGT_CUDA_TRY(cudaGetDevice(&dev));
    if (smem && !(attr_set.load() >> (dev & 63) & 1)) {
        EGT_CUDA_TRY(cudaFuncSetAttribute(k_knn_learned<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set.fetch_or(uint64_t(1) << (dev & 63));
    }
    unsigned G = 0;
    EGT_TRY(wave_blocks(k_knn_learned<S>, a.n, &G, smem));
    k_knn_learned<S><<<G, kWarps * 32, smem, st>>>(a, cls);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

// Largest cell population of each level (condition (4) above).
__global__ void k_maxpop(LevelDev lv0, LevelDev lv1, LevelDev lv2, LevelDev lv3, LevelDev lv4, LevelDev lv5,
                         LevelDev lv6, LevelDev lv7, int n, unsigned long long* __restrict__ counters) {
    const LevelDev* lvs[kMaxLevels] = {&lv0, &lv1, &lv2, &lv3, &lv4, &lv5, &lv6, &lv7};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int L = 0; L < kMaxLevels; L++) {
        const int nc = (int)counters[kCtrNcells + L];
        int v = (i < nc && i < n) ? lvs[L]->cell_start[i + 1] - lvs[L]->cell_start[i] : 0;
        v = __reduce_max_sync(0xffffffffu, v);
        if ((threadIdx.x & 31) == 0 && v > 0) atomicMax(&counters[kCtrMaxPop + L], (unsigned long long)v);
    }
}

template <int S, bool kFast>
egt_status launch(const KnnArgs& a, cudaStream_t st) {
    unsigned G = 0;
    EGT_TRY(wave_blocks(k_knn_plain<S, kFast>, a.n, &G));
    k_knn_plain<S, kFast><<<G, kWarps * 32, 0, st>>>(a);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

}  // namespace

egt_status level_maxpop(egt_handle* h) {
    if (h->maxpop_valid) return EGT_OK;
    cudaStream_t st = h->stream;
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrMaxPop, 0, kMaxLevels * sizeof(unsigned long long), st));
    const unsigned T = 256, G = (unsigned)((h->n + T - 1) / T);
    k_maxpop<<<G, T, 0, st>>>(h->lv[0], h->lv[1], h->lv[2], h->lv[3], h->lv[4], h->lv[5], h->lv[6], h->lv[7],
                              (int)h->n, h->d_counters);
    EGT_LAUNCH_CHECK();
    h->maxpop_valid = true;
    return EGT_OK;
}

// Lists and per-query buffers for k, and the search arguments of handle h.
static egt_status knn_prepare(egt_handle* h, int k, KnnArgs* a) {
    if (k <= 0 || k > 256) { set_error("egt_knn: k must be in [1, 256]"); return EGT_ERR_ARG; }
    if (h->levels_built < kMaxLevels) { set_error("egt_knn: grid hierarchy not built"); return EGT_ERR_STATE; }
    const int64_t n = h->n;
    if (h->k != k || !h->lists) {
        if (h->lists) dev_free(h, h->lists);
        h->lists = nullptr;
        EGT_CUDA_TRY(dev_alloc(h, &h->lists, sizeof(int) * (size_t)n * k));
        h->k = k;
    }
    if (!h->kth) EGT_CUDA_TRY(dev_alloc(h, &h->kth, sizeof(float) * n));
    if (!h->qlevel) EGT_CUDA_TRY(dev_alloc(h, &h->qlevel, n));
    h->have_csr = false;
    a->p4 = h->p4;
    a->np = h->d_norm;
    for (int L = 0; L < kMaxLevels; L++) a->lv[L] = h->lv[L];
    a->n = (int)n;
    a->k = k;
    a->max_pts = h->cfg.max_points_in_cell;
    a->chunk = kChunk;
    a->lists = h->lists;
    a->kth_out = h->kth;
    a->qlevel = h->qlevel;
    a->counters = h->d_counters;
    a->qmap = nullptr;
    return EGT_OK;
}

// One plain search launch over a.n queries (the work counter must be zero).
static egt_status knn_launch(const KnnArgs& a, cudaStream_t st) {
    const int k = a.k;
    // the list keeps k+1 slots (k for k = 256, which always uses the exact rule)
    if (k + 1 <= 32) EGT_TRY((launch<1, true>(a, st)));
    else if (k + 1 <= 64) EGT_TRY((launch<2, true>(a, st)));
    else if (k + 1 <= 96) EGT_TRY((launch<3, true>(a, st)));
    else if (k + 1 <= 128) EGT_TRY((launch<4, true>(a, st)));
    else if (k + 1 <= 256) EGT_TRY((launch<8, true>(a, st)));
    else EGT_TRY((launch<8, false>(a, st)));
    return EGT_OK;
}

template <typename K>
static egt_status select_blocks(K kernel, unsigned* out) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, unsigned> cache;
    int dev = 0;
    EGT_CUDA_TRY(cudaGetDevice(&dev));
    const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) { *out = it->second; return EGT_OK; }
    }
    int sms = 0, per = 0;
    EGT_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    EGT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kWarps * 32, 0));
    *out = (unsigned)std::max(1, sms * std::max(per, 1));
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = *out;
    return EGT_OK;
}

// Queries a warp of the selection kernel claims at a time: consecutive
// queries lie in nearby cells and mostly take the same level.
constexpr int kSelChunk = 16;

template <int S>
static egt_status launch_select(const KnnArgs& a, cudaStream_t st) {
    unsigned G = 0;
    EGT_TRY(select_blocks(k_knn_select<S>, &G));
    const int64_t need = ((int64_t)a.n + kWarps * a.chunk - 1) / (kWarps * a.chunk);
    G = (unsigned)std::max<int64_t>(1, std::min<int64_t>(G, need));
    k_knn_select<S><<<G, kWarps * 32, 0, st>>>(a);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

// The exact search of a.n queries (the work counter must be zero): the
// reference's ring search (k_knn_plain), or with `select` (EGT_KNN_SELECT, k <=
// kSelMaxK) the block-selection kernel, whose uncertified queries run the ring
// search in the same launch.
static egt_status knn_search(const KnnArgs& a, bool select, cudaStream_t st) {
    if (!select || a.k > kSelMaxK) return knn_launch(a, st);
    KnnArgs as = a;
    as.chunk = kSelChunk;
    if (a.k + 1 <= 32) return launch_select<1>(as, st);
    if (a.k + 1 <= 64) return launch_select<2>(as, st);
    return launch_select<3>(as, st);
}

// The cell-tile search of every query, then the ring search of the queries
// it could not certify (the counters must be reset).
static egt_status tile_search(egt_handle* h, const KnnArgs& a, cudaStream_t st) {
    TileArgs t;
    EGT_TRY(tile_prepare(h, &t));
    t.desc = nullptr;
    t.cloud_of = nullptr;
    t.npts = a.n;
    EGT_TRY(level_maxpop(h));  // condition (4)
    EGT_TRY(tile_launch<false>(a, t, a.k, st));
    KnnArgs ar = a;
    ar.qmap = t.ring2;
    ar.n_dev = t.n_ring2;
    ar.work = h->d_counters + kCtrTileRingWork;
    return knn_launch(ar, st);
}

egt_status run_knn(egt_handle* h, int k) {
    cudaStream_t st = h->stream;
    KnnArgs a;
    EGT_TRY(knn_prepare(h, k, &a));
    if (h->cfg.knn_mode == EGT_KNN_TILE && k >= kTileMinK && k <= kTileMaxK) {
        EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrInvalid, 0, 2 * sizeof(unsigned long long), st));
        EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrExactRerun, 0, 3 * sizeof(unsigned long long), st));
        EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrSelFallback, 0, sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrTileRing2, 0, sizeof(unsigned long long), st));
        EGT_CUDA_TRY(cudaEventRecord(h->ev[2], st));
        EGT_TRY(tile_search(h, a, st));
        EGT_CUDA_TRY(cudaEventRecord(h->ev[3], st));
        return EGT_OK;
    }
    const bool select = h->cfg.knn_mode == EGT_KNN_SELECT;
    if (select) EGT_TRY(level_maxpop(h));  // the selection's oversized-cell check
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrInvalid, 0, 2 * sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrExactRerun, 0, 3 * sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrSelFallback, 0, sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrTileRing2, 0, sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[2], st));
    EGT_TRY(knn_search(a, select, st));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[3], st));
    return EGT_OK;
}

namespace {
// Sort key of sorted slot s for the chunked search: the chunk of its original row.
constexpr int kMaxHostChunks = 16;
struct ChunkBounds {
    int end[kMaxHostChunks];  // chunk c holds the original rows [end[c-1], end[c])
    int count;
};

__global__ void k_chunk_keys(const int* __restrict__ perm, int n, ChunkBounds cb, uint32_t* __restrict__ key,
                             int* __restrict__ idx) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int r = perm[s];
    uint32_t c = 0;
    while ((int)c + 1 < cb.count && r >= cb.end[c]) c++;
    key[s] = c;
    idx[s] = s;
}

// Adds the per-chunk counts of uncertified queries to the handle's counter.
__global__ void k_sum_counts(const unsigned long long* __restrict__ v, int m, unsigned long long* __restrict__ out) {
    unsigned long long t = 0;
    for (int i = threadIdx.x; i < m; i += 32) t += v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) *out += t;
}

// Rows of queries qmap[0..m) in original order and ids (GetKNNIndexes layout).
__global__ void k_rows_original(const int* __restrict__ lists, const int* __restrict__ perm,
                                const int* __restrict__ qmap, int m, int k, int* __restrict__ out) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= (int64_t)m * k) return;
    const int j = (int)(e / k), t = (int)(e % k);
    const int q = qmap[j];
    const int v = lists[(size_t)q * k + t];
    out[(size_t)perm[q] * k + t] = v >= 0 ? perm[v] : -1;
}
}  // namespace

// The plain search with its lists delivered to the host in original order
// (egt_knn followed by egt_get_knn_host).  The queries are searched in chunks
// of original rows: the sorted slots are grouped by the chunk of their
// original row (a stable sort, so each chunk keeps sorted order and most of
// its spatial locality).  Chunks alternate between two streams, so one
// chunk's tail overlaps the next chunk's start, and each finished chunk's
// rows -- a contiguous block of the original-order output -- are copied to
// the host on a third stream while later chunks are searched.  The chunks
// shrink towards the end (20 % of the rows first, 1.5 % last): the copy of
// the last chunk is the part that nothing overlaps, and each copy still
// finishes before the next chunk's search (copying runs at about 0.6 of the
// search rate).  The handle's sorted-space lists are filled as egt_knn fills
// them.
egt_status run_knn_host(egt_handle* h, int k, int* host) {
    cudaStream_t st = h->stream;
    KnnArgs a;
    EGT_TRY(knn_prepare(h, k, &a));
    const int n = (int)h->n;
    ChunkBounds cb{};
    {
        static const double kShare[] = {0.2, 0.2, 0.2, 0.15, 0.1, 0.07, 0.04, 0.025, 0.015};
        const int parts = n >= 262144 ? (int)(sizeof(kShare) / sizeof(kShare[0])) : 1;
        double acc = 0.0;
        cb.count = 0;
        for (int c = 0; c < parts; c++) {
            acc += kShare[c];
            const int e = c == parts - 1 ? n : std::min(n, (int)(acc * n));
            if (cb.count > 0 && e <= cb.end[cb.count - 1]) continue;
            cb.end[cb.count++] = e;
        }
        if (parts == 1) cb.end[0] = n;
    }
    const int chunks = cb.count;
    int bits = 1;
    while ((1 << bits) < chunks) bits++;
    uint32_t *key = nullptr, *key2 = nullptr;
    int *idx = nullptr, *qmap = nullptr, *out = nullptr;
    unsigned long long* work = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&key, sizeof(uint32_t) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&key2, sizeof(uint32_t) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&idx, sizeof(int) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&qmap, sizeof(int) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&out, sizeof(int) * (size_t)n * k, st));
    // per chunk: its work counter and its count of queries the ring search ran
    EGT_CUDA_TRY(cudaMallocAsync((void**)&work, sizeof(unsigned long long) * 2 * chunks, st));
    EGT_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(unsigned long long) * 2 * chunks, st));
    if (h->cfg.knn_mode == EGT_KNN_SELECT) EGT_TRY(level_maxpop(h));
    const unsigned T = 256;
    k_chunk_keys<<<(unsigned)((n + T - 1) / T), T, 0, st>>>(h->perm, n, cb, key, idx);
    EGT_LAUNCH_CHECK();
    size_t t_sort = 0;
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, t_sort, key, key2, idx, qmap, n, 0, bits, st));
    void* tmp = nullptr;
    EGT_TRY(scratch_reserve(h, t_sort, &tmp));
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, t_sort, key, key2, idx, qmap, n, 0, bits, st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrInvalid, 0, 2 * sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrExactRerun, 0, sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrEvals, 0, sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrSelFallback, 0, sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrTileRing2, 0, sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[2], st));
    // streams: [0] = h->stream, [1] = a second search stream, [2] = copies
    cudaStream_t ss[3] = {st, nullptr, nullptr};
    std::vector<cudaEvent_t> ev(2 * chunks + 2, nullptr);
    egt_status s = EGT_OK;
    auto fail = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess && s == EGT_OK) { set_error(cuda_msg(e, what, __FILE__, __LINE__)); s = EGT_ERR_CUDA; }
    };
    fail(cudaStreamCreateWithFlags(&ss[1], cudaStreamNonBlocking), "cudaStreamCreate");
    fail(cudaStreamCreateWithFlags(&ss[2], cudaStreamNonBlocking), "cudaStreamCreate");
    for (size_t i = 0; i < ev.size() && s == EGT_OK; i++)
        fail(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming), "cudaEventCreate");
    // the second search stream starts after the set-up on the first
    if (s == EGT_OK) fail(cudaEventRecord(ev[2 * chunks], st), "cudaEventRecord");
    if (s == EGT_OK) fail(cudaStreamWaitEvent(ss[1], ev[2 * chunks], 0), "cudaStreamWaitEvent");
    for (int c = 0; c < chunks && s == EGT_OK; c++) {
        const int r0 = c == 0 ? 0 : cb.end[c - 1], m = cb.end[c] - r0;
        if (m <= 0) continue;
        cudaStream_t cs = ss[c & 1];
        // the chunk's sorted slots sit at qmap[r0, r0 + m): every chunk holds exactly its row count
        KnnArgs ac = a;
        ac.qmap = qmap + r0;
        ac.n = m;
        ac.work = work + c;
        ac.n_ring = work + chunks + c;
        s = knn_search(ac, h->cfg.knn_mode == EGT_KNN_SELECT, cs);
        if (s != EGT_OK) break;
        const int64_t cnt = (int64_t)m * k;
        k_rows_original<<<(unsigned)((cnt + T - 1) / T), T, 0, cs>>>(h->lists, h->perm, qmap + r0, m, k, out);
        count_launch();
        fail(cudaGetLastError(), "k_rows_original");
        if (s == EGT_OK) fail(cudaEventRecord(ev[c], cs), "cudaEventRecord");
        if (s == EGT_OK) fail(cudaStreamWaitEvent(ss[2], ev[c], 0), "cudaStreamWaitEvent");
        if (s == EGT_OK)
            fail(cudaMemcpyAsync(host + (size_t)r0 * k, out + (size_t)r0 * k, sizeof(int) * cnt,
                                 cudaMemcpyDeviceToHost, ss[2]),
                 "chunk copy");
    }
    // join: the first stream waits for the second search stream, then ends the timing
    if (s == EGT_OK) fail(cudaEventRecord(ev[2 * chunks + 1], ss[1]), "cudaEventRecord");
    if (s == EGT_OK) fail(cudaStreamWaitEvent(st, ev[2 * chunks + 1], 0), "cudaStreamWaitEvent");
    if (s == EGT_OK) {
        k_sum_counts<<<1, 32, 0, st>>>(work + chunks, chunks, h->d_counters + kCtrSelFallback);
        count_launch();
        fail(cudaGetLastError(), "k_sum_counts");
    }
    if (s == EGT_OK) fail(cudaEventRecord(h->ev[3], st), "cudaEventRecord");
    fail(cudaStreamSynchronize(ss[2]), "copy stream");
    fail(cudaStreamSynchronize(ss[1]), "search stream");
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    if (ss[1]) cudaStreamDestroy(ss[1]);
    if (ss[2]) cudaStreamDestroy(ss[2]);
    cudaFreeAsync(key, st); cudaFreeAsync(key2, st); cudaFreeAsync(idx, st); cudaFreeAsync(qmap, st);
    cudaFreeAsync(out, st); cudaFreeAsync(work, st);
    fail(cudaStreamSynchronize(st), "stream");
    return s;
}

template <int S>
static egt_status launch_query(const KnnArgs& a, const float4* qpos, const int* perm, int* out, cudaStream_t st) {
    unsigned G = 0;
    EGT_TRY(wave_blocks(k_knn_query<S>, a.n, &G));
    k_knn_query<S><<<G, kWarps * 32, 0, st>>>(a, qpos, perm, out);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

// Query-vs-reference kNN against handle h's grid (GRIDCUDAKNNCompact +
// GetKNNIndexes): q_host [nq*3] AoS query points in the reference's units,
// out_host [nq*k] original reference ids in original query order.  The
// handle's own lists and statistics are untouched.  Queries are processed in
// the order of their level-0 cell (the reference also sorts them by cell,
// GridKNNCuda.cu:1208-1267; the order does not change any result).
egt_status run_knn_query(egt_handle* h, const float* q_host, int64_t nq, int k, int* out_host, int64_t* invalid) {
    if (k <= 0 || k > 255) { set_error("egt_knn_query: k must be in [1, 255]"); return EGT_ERR_ARG; }
    if (nq < 0 || nq > 0x7fffffff || (nq > 0 && (!q_host || !out_host))) {
        set_error("egt_knn_query: bad query arguments");
        return EGT_ERR_ARG;
    }
    if ((int64_t)k * nq > (int64_t)0x7fffffff) { set_error("egt_knn_query: nq*k exceeds 2^31-1"); return EGT_ERR_ARG; }
    if (h->levels_built < kMaxLevels) { set_error("egt_knn_query: grid hierarchy not built"); return EGT_ERR_STATE; }
    if (invalid) *invalid = 0;
    if (nq == 0) return EGT_OK;
    cudaStream_t st = h->stream;
    const int n = (int)nq;
    float* dq = nullptr;
    float4* qpos = nullptr;
    uint32_t *key = nullptr, *key2 = nullptr;
    int *idx = nullptr, *qmap = nullptr, *out = nullptr;
    unsigned long long* ctr = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&dq, sizeof(float) * 3 * (size_t)n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&qpos, sizeof(float4) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&key, sizeof(uint32_t) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&key2, sizeof(uint32_t) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&idx, sizeof(int) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&qmap, sizeof(int) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&out, sizeof(int) * (size_t)n * k, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&ctr, sizeof(unsigned long long) * kCtrWords, st));
    EGT_CUDA_TRY(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long) * kCtrWords, st));
    EGT_CUDA_TRY(cudaMemcpyAsync(dq, q_host, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, st));
    const unsigned T = 256;
    k_query_prepare<<<(unsigned)((n + T - 1) / T), T, 0, st>>>(dq, n, h->d_norm, qpos, key, idx);
    EGT_LAUNCH_CHECK();
    size_t t_sort = 0;
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, t_sort, key, key2, idx, qmap, n, 0, 30, st));
    void* tmp = nullptr;
    EGT_TRY(scratch_reserve(h, t_sort, &tmp));
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, t_sort, key, key2, idx, qmap, n, 0, 30, st));
    KnnArgs a;
    a.p4 = h->p4;
    a.np = h->d_norm;
    for (int L = 0; L < kMaxLevels; L++) a.lv[L] = h->lv[L];
    a.n = n;
    a.k = k;
    a.max_pts = h->cfg.max_points_in_cell;
    a.chunk = kChunk;
    a.lists = nullptr;
    a.kth_out = nullptr;
    a.qlevel = nullptr;
    a.counters = ctr;
    a.qmap = qmap;
    egt_status s;
    if (k + 1 <= 32) s = launch_query<1>(a, qpos, h->perm, out, st);
    else if (k + 1 <= 64) s = launch_query<2>(a, qpos, h->perm, out, st);
    else if (k + 1 <= 96) s = launch_query<3>(a, qpos, h->perm, out, st);
    else if (k + 1 <= 128) s = launch_query<4>(a, qpos, h->perm, out, st);
    else s = launch_query<8>(a, qpos, h->perm, out, st);
    unsigned long long inv = 0;
    if (s == EGT_OK) {
        cudaError_t e = cudaMemcpyAsync(out_host, out, sizeof(int) * (size_t)n * k, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&inv, ctr + kCtrInvalid, sizeof(inv), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) { set_error(cuda_msg(e, "query results", __FILE__, __LINE__)); s = EGT_ERR_CUDA; }
    }
    cudaFreeAsync(dq, st); cudaFreeAsync(qpos, st); cudaFreeAsync(key, st); cudaFreeAsync(key2, st);
    cudaFreeAsync(idx, st); cudaFreeAsync(qmap, st); cudaFreeAsync(out, st); cudaFreeAsync(ctr, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess && s == EGT_OK) { set_error(cuda_msg(e, "egt_knn_query", __FILE__, __LINE__)); s = EGT_ERR_CUDA; }
    if (s == EGT_OK && invalid) *invalid = (int64_t)inv;
    return s;
}

egt_status run_knn_learned(egt_handle* h, int k, const egt_proposal* p) {
    if (k <= 0 || k > 255) { set_error("egt_knn_learned: k must be in [1, 255]"); return EGT_ERR_ARG; }
    if (h->levels_built < kMaxLevels) { set_error("egt_knn_learned: grid hierarchy not built"); return EGT_ERR_STATE; }
    cudaStream_t st = h->stream;
    const int64_t n = h->n;
    if (h->k != k || !h->lists) {
        if (h->lists) dev_free(h, h->lists);
        h->lists = nullptr;
        EGT_CUDA_TRY(dev_alloc(h, &h->lists, sizeof(int) * (size_t)n * k));
        h->k = k;
    }
    if (!h->kth) EGT_CUDA_TRY(dev_alloc(h, &h->kth, sizeof(float) * n));
    if (!h->qlevel) EGT_CUDA_TRY(dev_alloc(h, &h->qlevel, n));
    h->have_csr = false;
    EGT_CUDA_TRY(cudaEventRecord(h->ev[2], st));
    EGT_TRY(level_maxpop(h));
    EGT_TRY(proposal_classes(h, p));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[15], st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrInvalid, 0, 2 * sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrBoxTried, 0, 2 * sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrExactRerun, 0, 3 * sizeof(unsigned long long), st));
    KnnArgs a;
    a.p4 = h->p4;
    a.np = h->d_norm;
    for (int L = 0; L < kMaxLevels; L++) a.lv[L] = h->lv[L];
    a.n = (int)n;
    a.k = k;
    a.max_pts = h->cfg.max_points_in_cell;
    a.chunk = kChunk;
    a.lists = h->lists;
    a.kth_out = h->kth;
    a.qlevel = h->qlevel;
    a.counters = h->d_counters;
    if (k + 1 <= 32) EGT_TRY(launch_learned<1>(a, h->pclass, st));
    else if (k + 1 <= 64) EGT_TRY(launch_learned<2>(a, h->pclass, st));
    else if (k + 1 <= 96) EGT_TRY(launch_learned<3>(a, h->pclass, st));
    else if (k + 1 <= 128) EGT_TRY(launch_learned<4>(a, h->pclass, st));
    else EGT_TRY(launch_learned<8>(a, h->pclass, st));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[3], st));
    h->tm.propose_ms = -1.0f;  // filled from the events by egt_get_timings
    return EGT_OK;
}

}  // namespace egt
