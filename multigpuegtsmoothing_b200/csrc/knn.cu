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
#include <map>
#include <mutex>

#include "egt_internal.cuh"
#include "knn_common.cuh"
#include "proposal.cuh"

namespace egt {
namespace {

struct KnnArgs {
    const float4* __restrict__ p4;
    const NormParams* __restrict__ np;
    LevelDev lv[kMaxLevels];
    int n, k, max_pts;
    int* __restrict__ lists;
    float* __restrict__ kth_out;
    uint8_t* __restrict__ qlevel;
    unsigned long long* __restrict__ counters;
};

constexpr int kWarps = 8;

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

// Batches admitting at least this many candidates are merged in one step.
constexpr int kMergeMin = 3;

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
    if (!kExact && __popc(mask) >= kMergeMin) {
        merge_batch(L, d, p, adm, lane, s_md, s_mp);
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

// Streams the points of `m` cells (cell l held by lane l as [cs, ce), ce < 0 =
// empty) through the list, in cell order.  Sets `invalid` when a visited cell
// holds >= max_pts points (GridKNNCuda.cu:672, 685): the cells before it are
// still processed, the rest are not.  skipL >= 0: skip points whose level-skipL
// cell lies in the 3x3x3 block around the query's (already visited).
template <bool kExact, int S>
__device__ __forceinline__ void stream_cells(WarpList<S>& L, bool& invalid, int m, int cs, int ce,
                                             const int* __restrict__ order, const float4* __restrict__ p4,
                                             int q, float4 pq, float thres, int max_pts, int lane,
                                             int skipL, uint32_t qc0, int* s_pref, int* s_start, float* s_md,
                                             int* s_mp) {
    const bool exists = lane < m && ce >= 0;
    const bool big = exists && (ce - cs) >= max_pts;
    const unsigned bigmask = __ballot_sync(0xffffffffu, big);
    const int mlim = bigmask ? (__ffs(bigmask) - 1) : m;
    int sz = (lane < mlim && exists) ? ce - cs : 0;
    int incl = sz;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    __syncwarp();
    s_pref[lane] = incl;
    s_start[lane] = cs;
    __syncwarp();
    const int qx = (int)((qc0 & 1023u) >> max(skipL, 0)), qy = (int)(((qc0 >> 10) & 1023u) >> max(skipL, 0)),
              qz = (int)(((qc0 >> 20) & 1023u) >> max(skipL, 0));
    for (int base = 0; base < total; base += 32) {
        const int j = base + lane;
        float d = 1e30f;
        int p = -1;
        bool ok = false;
        if (j < total) {
            int lo = 0, hi = mlim - 1;  // first cell with incl > j
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (s_pref[mid] > j) hi = mid;
                else lo = mid + 1;
            }
            const int excl = lo > 0 ? s_pref[lo - 1] : 0;
            const int pos = s_start[lo] + (j - excl);
            p = order ? order[pos] : pos;
            if (p != q) {
                const float4 v = p4[p];
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
                }
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
    stream_cells<kExact, S>(L, invalid, 1, own.x, own.y, nullptr, a.p4, q, pq, np.thres, a.max_pts, lane, -1, c0,
                            s_pref, s_start, s_md, s_mp);
    bool cont = decide(np, 0, 0, L.counter, k, kExact ? L.kth : L.fetch_dist(k - 1), invalid, pq, cx0, cy0, cz0);
    int reached = 0;
    for (int lvl = 0; cont; lvl++) {
        reached = lvl;
        const LevelDev& LV = a.lv[lvl];
        int2 cell = make_int2(-1, -1);
        if (lane < 26)
            cell = find_cell(LV, (cx0 >> lvl) + kShell[lane][0], (cy0 >> lvl) + kShell[lane][1],
                             (cz0 >> lvl) + kShell[lane][2]);
        stream_cells<kExact, S>(L, invalid, 26, cell.x, cell.y, LV.order, a.p4, q, pq, np.thres, a.max_pts, lane,
                                lvl - 1, c0, s_pref, s_start, s_md, s_mp);
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

// Queries claimed per atomic by a warp of the persistent kNN kernels.
constexpr int kChunk = 4;

// Next chunk of queries for the calling warp (uniform); >= n when done.
__device__ __forceinline__ int claim(const KnnArgs& a, int lane) {
    unsigned long long q0 = 0;
    if (lane == 0) q0 = atomicAdd(&a.counters[kCtrWork], (unsigned long long)kChunk);
    return (int)min(__shfl_sync(0xffffffffu, q0, 0), (unsigned long long)a.n);
}

// Persistent: one resident wave of blocks whose warps claim kChunk queries at
// a time, so that a warp that drew cheap queries moves on instead of idling
// until the most expensive query of its block is done.
template <int S, bool kFast>
__global__ void __launch_bounds__(kWarps * 32) k_knn_plain(KnnArgs a) {
    __shared__ int s_pref[kWarps][32];
    __shared__ int s_start[kWarps][32];
    __shared__ float s_md[kWarps][32 * S];
    __shared__ int s_mp[kWarps][32 * S];
    __shared__ unsigned s_rerun;
    if (threadIdx.x == 0) s_rerun = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const NormParams np = *a.np;
    for (int q0 = claim(a, lane); q0 < a.n; q0 = claim(a, lane)) {
        const int q1 = min(q0 + kChunk, a.n);
        for (int q = q0; q < q1; q++) {
            const float4 pq = a.p4[q];
            WarpList<S> L;
            bool invalid, rerun;
            const int reached = plain_query<kFast, S>(a, np, q, pq, L, invalid, lane, s_pref[w], s_start[w], s_md[w],
                                                      s_mp[w], rerun);
            write_query<S>(a, q, L, invalid, reached, lane);
            if (rerun && lane == 0) atomicAdd(&s_rerun, 1u);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_rerun) atomicAdd(&a.counters[kCtrExactRerun], (unsigned long long)s_rerun);
}

// ---------------------------------------------------------------------------
// Proposal-driven search (an extension of this project).  The query's box
// (class from the proposal network) is streamed row by row, nearest rows
// first, keeping the k+1 smallest distances.  The result is accepted only when
// it provably equals the plain search's list:
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
// The box may be cut short after any complete ring of rows whose sub-box
// already passes (2).  A failed check runs the plain search for the query.

// Streams the points of m row ranges (range l held by lane l as [cs, ce)).
template <int S>
__device__ __forceinline__ void stream_ranges(WarpList<S>& L, int m, int cs, int ce, const int* __restrict__ order,
                                              const float4* __restrict__ p4, int q, float4 pq, float thres, int lane,
                                              int* s_pref, int* s_start, float* s_md, int* s_mp) {
    int incl = lane < m ? ce - cs : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    __syncwarp();
    s_pref[lane] = incl;
    s_start[lane] = cs;
    __syncwarp();
    for (int base = 0; base < total; base += 32) {
        const int j = base + lane;
        float d = 1e30f;
        int p = -1;
        bool ok = false;
        if (j < total) {
            int lo = 0, hi = m - 1;  // first range with incl > j
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (s_pref[mid] > j) hi = mid;
                else lo = mid + 1;
            }
            const int excl = lo > 0 ? s_pref[lo - 1] : 0;
            const int pos = s_start[lo] + (j - excl);
            p = order ? order[pos] : pos;
            if (p != q) {
                const float4 v = p4[p];
                d = fs_dist3(pq.x, pq.y, pq.z, v.x, v.y, v.z);
                ok = d <= thres;
            }
        }
        offer<false, S>(L, d, p, ok && d < L.kth, lane, s_md, s_mp);
    }
}

// Box search + certification.  Returns true with L holding the plain
// search's list in slots [0, k) and `reached` its level.
template <int S>
__device__ bool box_search(const KnnArgs& a, const NormParams& np, int q, float4 pq, int cls, WarpList<S>& L,
                           int lane, int* s_pref, int* s_start, float* s_md, int* s_mp, int& reached) {
    const int lvl = kBoxClass[cls][0], R = kBoxClass[cls][1];
    const LevelDev& LV = a.lv[lvl];
    const uint32_t c0 = __float_as_uint(pq.w);
    const int cx0 = c0 & 1023u, cy0 = (c0 >> 10) & 1023u, cz0 = (c0 >> 20) & 1023u;
    const int cix = cx0 >> lvl, ciy = cy0 >> lvl, ciz = cz0 >> lvl;
    const int k = a.k;
    L.init(k + 1);
    const int nrows = (2 * R + 1) * (2 * R + 1);
    int ring = -1;
    bool inside = false;
    for (int rb = 0; rb < nrows && !inside; rb += 32) {
        int2 rg = make_int2(0, 0);
        const int t = rb + lane;
        if (t < nrows) rg = row_points(LV, cix - R, cix + R, ciy + kRowOrder[t][0], ciz + kRowOrder[t][1]);
        stream_ranges<S>(L, min(32, nrows - rb), rg.x, rg.y, lvl ? LV.order : nullptr, a.p4, q, pq, np.thres, lane,
                         s_pref, s_start, s_md, s_mp);
        // largest ring of rows completely streamed
        const int done = min(rb + 32, nrows);
        int j = ring;
        while ((2 * j + 3) * (2 * j + 3) <= done) j++;
        if (j > ring) {
            ring = j;
            if (L.counter >= k) {
                int lo[3], end[3];
                box_bounds(cls, ring, c0, lo, end);
                inside = ball_in_box(np, pq, L.fetch_dist(k - 1), lo, end);  // (2)
            }
        }
    }
    if (!inside) return false;
    // (1) the kept distances are strictly increasing
    if (has_ties(L, min(L.counter, k + 1), lane)) return false;
    const float kth = L.fetch_dist(k - 1);
    // (3) the plain stop step, and the step by which G is visited
    int sg = 0;
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        if (t < k) sg = max(sg, visit_step(__float_as_uint(a.p4[L.idx[s]].w), c0));
    }
    sg = __reduce_max_sync(0xffffffffu, sg);
    int sf = -1;
    for (int st = 0; st <= kMaxLevels; st++) {
        const int Ls = st == 0 ? 0 : st - 1, o = st == 0 ? 0 : 1;
        if (!decide(np, Ls, o, k, k, kth, false, pq, cx0, cy0, cz0)) { sf = st; break; }
        if (!decide(np, Ls, o, 0, k, kth, false, pq, cx0, cy0, cz0)) return false;
    }
    if (sf < 0 || sg > sf) return false;
    // (4) no oversized cell on the visited levels
    for (int l = 0; l <= max(sf - 1, 0); l++)
        if (a.counters[kCtrMaxPop + l] >= (unsigned long long)a.max_pts) return false;
    reached = max(sf - 1, 0);
    return true;
}

template <int S>
__global__ void __launch_bounds__(kWarps * 32) k_knn_learned(KnnArgs a, const uint8_t* __restrict__ cls) {
    __shared__ int s_pref[kWarps][32];
    __shared__ int s_start[kWarps][32];
    __shared__ float s_md[kWarps][32 * S];
    __shared__ int s_mp[kWarps][32 * S];
    __shared__ unsigned s_box, s_cert, s_rerun;
    if (threadIdx.x == 0) { s_box = 0; s_cert = 0; s_rerun = 0; }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const NormParams np = *a.np;
    for (int q0 = claim(a, lane); q0 < a.n; q0 = claim(a, lane)) {
        const int q1 = min(q0 + kChunk, a.n);
        for (int q = q0; q < q1; q++) {
            const float4 pq = a.p4[q];
            WarpList<S> L;
            bool invalid = false, ok = false;
            int reached = 0;
            const int c = cls[q];
            if (c < kPropPlain) {
                ok = box_search<S>(a, np, q, pq, c, L, lane, s_pref[w], s_start[w], s_md[w], s_mp[w], reached);
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

// Blocks of one resident wave of a persistent kernel, per (kernel, device).
template <typename K>
egt_status wave_blocks(K kernel, int64_t n, unsigned* out) {
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
        EGT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kWarps * 32, 0));
        blocks = std::max(1, sms * std::max(per, 1));
        std::lock_guard<std::mutex> lock(mu);
        cache[key] = blocks;
    }
    const int64_t need = (n + kWarps * kChunk - 1) / (kWarps * kChunk);
    *out = (unsigned)std::max<int64_t>(1, std::min<int64_t>(blocks, need));
    return EGT_OK;
}

template <int S>
egt_status launch_learned(const KnnArgs& a, const uint8_t* cls, cudaStream_t st) {
    unsigned G = 0;
    EGT_TRY(wave_blocks(k_knn_learned<S>, a.n, &G));
    k_knn_learned<S><<<G, kWarps * 32, 0, st>>>(a, cls);
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

egt_status run_knn(egt_handle* h, int k) {
    if (k <= 0 || k > 256) { set_error("egt_knn: k must be in [1, 256]"); return EGT_ERR_ARG; }
    if (h->levels_built < kMaxLevels) { set_error("egt_knn: grid hierarchy not built"); return EGT_ERR_STATE; }
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
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrInvalid, 0, 2 * sizeof(unsigned long long), st));
    KnnArgs a;
    a.p4 = h->p4;
    a.np = h->d_norm;
    for (int L = 0; L < kMaxLevels; L++) a.lv[L] = h->lv[L];
    a.n = (int)n;
    a.k = k;
    a.max_pts = h->cfg.max_points_in_cell;
    a.lists = h->lists;
    a.kth_out = h->kth;
    a.qlevel = h->qlevel;
    a.counters = h->d_counters;
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrExactRerun, 0, 2 * sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[2], st));
    // the list keeps k+1 slots (k for k = 256, which always uses the exact rule)
    if (k + 1 <= 32) EGT_TRY((launch<1, true>(a, st)));
    else if (k + 1 <= 64) EGT_TRY((launch<2, true>(a, st)));
    else if (k + 1 <= 96) EGT_TRY((launch<3, true>(a, st)));
    else if (k + 1 <= 128) EGT_TRY((launch<4, true>(a, st)));
    else if (k + 1 <= 256) EGT_TRY((launch<8, true>(a, st)));
    else EGT_TRY((launch<8, false>(a, st)));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[3], st));
    return EGT_OK;
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
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrExactRerun, 0, 2 * sizeof(unsigned long long), st));
    KnnArgs a;
    a.p4 = h->p4;
    a.np = h->d_norm;
    for (int L = 0; L < kMaxLevels; L++) a.lv[L] = h->lv[L];
    a.n = (int)n;
    a.k = k;
    a.max_pts = h->cfg.max_points_in_cell;
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
