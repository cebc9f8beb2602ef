// Exact self-kNN by block selection: the fast path of egt_knn.
//
// The reference's ring search (GRIDCUDAKNNSELF_COMPACT, GridKNNCuda.cu:2322-2634,
// with its stop rule construct_neighbors_self_compact, :694-741) is an exact
// k-nearest-neighbour search: step 0 visits the query's own level-0 cell, step
// s >= 1 the 3x3x3 block of level-(s-1) cells around it, and the search stops
// at the first step whose k-th distance r satisfies sqrt(r) < the distance to
// every in-grid face of that block.  If the k nearest points of the whole
// cloud lie inside the block of a step and their k-th distance T passes that
// step's face test, the step's k-th distance is T and the search stops there;
// at every earlier step its k-th distance is >= T, so it fails the face test
// wherever T fails it.  The reference's list is then the cloud's k nearest
// points in ascending distance -- provided the k+1 smallest distances are
// pairwise distinct, since the order of equal distances follows the reference's
// insertion rule (FindPosition, GridKNNCuda.cu:126-143) and the candidate
// order, and no cell the search visits holds max_points_in_cell points or more
// (such a cell invalidates the query, GridKNNCuda.cu:672, 685).
//
// So one warp per query:
//   1. gathers the 3x3x3 block of level-G cells around the query (G from the
//      previous query of the warp, one lower when that block holds 4(k+1)
//      points) as one flattened candidate sequence, 32 per step;
//   2. completeness: every point of the cloud within (nearest in-grid block
//      face - 2e-6) of the query lies in the block (the margin covers the float
//      rounding of cell keys and distances), so the block's points below that
//      bound are all such points of the cloud;
//   3. pass 1 computes every distance (the reference's contracted form), keeps
//      it in shared memory and counts those below the bound into 64 linear
//      buckets; fewer than k+1 below the bound: next level; else a warp scan
//      finds the bucket of the (k+1)-th smallest and pass 2 collects that
//      bucket and the lower ones;
//   4. sorts the collected candidates (warp bitonic sort): their k+1 smallest
//      are the cloud's k+1 nearest points;
//   5. certifies the result: k+1 distinct distances; the stop step s* of the
//      reference replayed with its own face test (decide) on T; the k nearest
//      inside the block of step s* (their cell keys); no oversized cell on the
//      levels up to s*.  A certified query's row is written.  Any other query
//      runs the ring search (the exact insertion rule included) in the same
//      warp.
// The lists are therefore bit-identical to the ring search's, tie order
// included.  A candidate costs a distance, a bucket count and a shared-memory
// store instead of a list merge, but the whole block is evaluated, about 2.3
// times the candidates the ring search's per-level culling evaluates on the
// 4M-point superquadric workload; there the ring search is faster and is
// egt_knn's default (this path is EGT_KNN_SELECT).
#pragma once
#include <climits>
#include "egt_internal.cuh"
#include "knn_common.cuh"
#include "knn_search.cuh"
#include "proposal.cuh"

namespace egt {
namespace {

constexpr int kSelBuckets = 64;   // linear distance buckets below the completeness bound
constexpr int kSelCollect = 128;  // collected candidates per query (the (k+1)-th's bucket and below)
constexpr int kSelCache = 1024;   // candidate distances kept between the two passes
constexpr int kSelMaxK = 95;      // k + 1 <= 96 leaves room in the collection for the boundary bucket

// Per-warp shared scratch of the selection kernel (16-byte aligned: a fused
// filter stages float4 positions in `d`).
struct alignas(16) SelScratch {
    float d[kSelCache];
    int hist[kSelBuckets];
    float cd[kSelCollect];
    int cj[kSelCollect];
    int pref[32];
    int start[32];
};

// Squared-distance bound below which every point of the cloud lies in the
// 3x3x3 block of level-L cells around level-0 cell c0: (nearest in-grid block
// face - margin)^2, rounded down; 3e38 when no face of the block is inside the
// grid.  The faces are placed as ball_in_box places them (double arithmetic on
// the exact level-0 cell width).
__device__ __forceinline__ float block_bound(const NormParams& np, float4 pq, int L, uint32_t c0) {
    const int ci[3] = {(int)(c0 & 1023u) >> L, (int)((c0 >> 10) & 1023u) >> L, (int)((c0 >> 20) & 1023u) >> L};
    const double h0 = (double)__fmul_rn(__fsub_rn(np.b, np.a), 1.0f / 1024.0f);
    const double c[3] = {pq.x, pq.y, pq.z};
    double fnear = 1e30;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const int lo = (ci[d] - 1) << L, end = (ci[d] + 2) << L;
        if (lo > 0) fnear = fmin(fnear, c[d] - ((double)np.a + lo * h0));
        if (end < 1024) fnear = fmin(fnear, ((double)np.a + end * h0) - c[d]);
    }
    if (fnear >= 1e29) return 3.0e38f;
    const double t = fnear - kBoxMargin;
    return t > 0.0 ? __double2float_rd(t * t) : 0.0f;
}

// Bucket of a distance below the bound: monotone in d.
__device__ __forceinline__ int sel_bucket(float d, float scale) {
    return min((int)__fmul_rz(d, scale), kSelBuckets - 1);
}

// (d, j) strictly before (e, k)
__device__ __forceinline__ bool sel_less(float d, int j, float e, int k) { return d < e || (d == e && j < k); }

// Ascending warp bitonic sort of 32*R (distance, position) pairs; element e
// is register e / 32 of lane e % 32.
template <int R>
__device__ __forceinline__ void sel_sort(float (&d)[R], int (&j)[R], int lane) {
    constexpr int N = 32 * R;
#pragma unroll
    for (int size = 2; size <= N; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (stride >= 32) {
                const int rs = stride >> 5;
#pragma unroll
                for (int r = 0; r < R; r++) {
                    const int r2 = r ^ rs;
                    if (r2 > r) {
                        const bool up = ((r * 32 + lane) & size) == 0;
                        const bool sw = up ? sel_less(d[r2], j[r2], d[r], j[r]) : sel_less(d[r], j[r], d[r2], j[r2]);
                        if (sw) {
                            const float td = d[r]; d[r] = d[r2]; d[r2] = td;
                            const int tj = j[r]; j[r] = j[r2]; j[r2] = tj;
                        }
                    }
                }
            } else {
#pragma unroll
                for (int r = 0; r < R; r++) {
                    const float od = __shfl_xor_sync(0xffffffffu, d[r], stride);
                    const int oj = __shfl_xor_sync(0xffffffffu, j[r], stride);
                    const bool up = ((r * 32 + lane) & size) == 0;
                    const bool keep_min = ((lane & stride) == 0) == up;
                    const bool take = keep_min ? sel_less(od, oj, d[r], j[r]) : sel_less(d[r], j[r], od, oj);
                    if (take) { d[r] = od; j[r] = oj; }
                }
            }
        }
    }
}

// Element e (uniform) of a sorted register array.
template <int R>
__device__ __forceinline__ float sel_at(const float (&d)[R], int e) {
    float v = d[0];
#pragma unroll
    for (int r = 1; r < R; r++)
        if ((e >> 5) == r) v = d[r];
    return __shfl_sync(0xffffffffu, v, e & 31);
}

// Result of one query: the sorted-space indices of its k nearest (slot t in
// register t / 32 of lane t % 32), their k-th distance and the reference's
// stop level; or not certified.
struct SelOut {
    bool ok;
    int reached;
    float kth;
};

// Sorts the collected candidates, certifies them and, when certified, writes
// query q's row.  c = collected count (k+1 <= c <= kSelCollect).
template <int R>
__device__ __noinline__ SelOut sel_finish(const KnnArgs& a, const NormParams& np, int q, float4 pq, int G, int lane,
                                             const SelScratch& sc, int c, const RangeSeq& seq) {
    SelOut out{false, 0, 0.0f};
    const int k = a.k;
    float d[R];
    int j[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int e = r * 32 + lane;
        d[r] = e < c ? sc.cd[e] : 3.4e38f;
        j[r] = e < c ? sc.cj[e] : INT_MAX;
    }
    sel_sort<R>(d, j, lane);
    // (1) the k+1 smallest distances pairwise distinct
    bool tie = false;
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int e = r * 32 + lane;
        const float up = __shfl_up_sync(0xffffffffu, d[r], 1);
        const float wrap = __shfl_sync(0xffffffffu, r > 0 ? d[r > 0 ? r - 1 : 0] : 0.f, 31);
        const float prev = lane == 0 ? wrap : up;
        if (e >= 1 && e <= k && !(prev < d[r])) tie = true;
    }
    if (__any_sync(0xffffffffu, tie)) return out;
    const float kth = sel_at<R>(d, k - 1);
    // (2) the reference's stop step for k-th distance kth: lane s replays step s
    const uint32_t c0 = __float_as_uint(pq.w);
    const int cx0 = c0 & 1023u, cy0 = (c0 >> 10) & 1023u, cz0 = (c0 >> 20) & 1023u;
    bool stop = false;
    if (lane <= kMaxLevels) {
        const int Ls = lane == 0 ? 0 : lane - 1, o = lane == 0 ? 0 : 1;
        stop = !decide(np, Ls, o, k, k, kth, false, pq, cx0, cy0, cz0);
    }
    const unsigned sm = __ballot_sync(0xffffffffu, stop);
    if (!sm) return out;  // still searching after the last level: the ring search decides
    const int sf = __ffs(sm) - 1;
    // (3) sequence position -> sorted index, and the k nearest inside step sf's block
    int idx[R];
    bool inside = true;
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int e = r * 32 + lane;
        idx[r] = -1;
        if (e < k) {
            int lo = 0, hi = seq.m - 1;  // first range whose inclusive end exceeds j
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (sc.pref[mid] <= j[r]) lo = mid + 1;
                else hi = mid;
            }
            const int prev_end = lo > 0 ? sc.pref[lo - 1] : 0;
            const int pos = sc.start[lo] + (j[r] - prev_end);
            idx[r] = G ? __ldg(a.lv[G].order + pos) : pos;
            inside &= visit_step(__float_as_uint(__ldg(&a.p4[idx[r]].w)), c0) <= sf;
        }
    }
    if (!__all_sync(0xffffffffu, inside)) return out;
    // (4) no oversized cell on the levels the reference visits up to step sf
    for (int l = 0; l <= max(sf - 1, 0); l++)
        if (a.counters[kCtrMaxPop + l] >= (unsigned long long)a.max_pts) return out;
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int e = r * 32 + lane;
        if (e < k) a.lists[(size_t)q * k + e] = idx[r];
    }
    out.ok = true;
    out.reached = max(sf - 1, 0);
    out.kth = kth;
    return out;
}

// The selection search of query q (see the file comment).  gstart: level to
// try first (updated to the level that resolved the query).  evals: candidate
// distances computed by this lane.
__device__ SelOut sel_query(const KnnArgs& a, const NormParams& np, int q, float4 pq, int lane, SelScratch& sc,
                            int& gstart, unsigned& evals) {
    SelOut fail{false, 0, 0.0f};
    const uint32_t c0 = __float_as_uint(pq.w);
    const int cx0 = c0 & 1023u, cy0 = (c0 >> 10) & 1023u, cz0 = (c0 >> 20) & 1023u;
    const int k = a.k;
    int G = gstart;
    // a level lower than the last one when it holds plenty of candidates
    if (G > 0) {
        const LevelDev& LV = a.lv[G - 1];
        int sz = 0;
        if (lane < 27) {
            const int dx = lane < 26 ? kShell[lane][0] : 0, dy = lane < 26 ? kShell[lane][1] : 0,
                      dz = lane < 26 ? kShell[lane][2] : 0;
            const int2 cell = find_cell(LV, (cx0 >> (G - 1)) + dx, (cy0 >> (G - 1)) + dy, (cz0 >> (G - 1)) + dz);
            sz = cell.x >= 0 ? cell.y - cell.x : 0;
        }
        if (__reduce_add_sync(0xffffffffu, sz) >= 4 * (k + 1)) G--;
    }
    for (; G < kMaxLevels; G++) {
        const LevelDev& LV = a.lv[G];
        int2 cell = make_int2(-1, -1);
        if (lane < 27) {
            const int dx = lane < 26 ? kShell[lane][0] : 0, dy = lane < 26 ? kShell[lane][1] : 0,
                      dz = lane < 26 ? kShell[lane][2] : 0;
            cell = find_cell(LV, (cx0 >> G) + dx, (cy0 >> G) + dy, (cz0 >> G) + dz);
        }
        const int sz = cell.x >= 0 ? cell.y - cell.x : 0;
        if (__reduce_add_sync(0xffffffffu, sz) < k + 2) continue;  // fewer than k+1 other points
        const float bound = block_bound(np, pq, G, c0);
        const float scale = __fdiv_rz((float)kSelBuckets, fmaxf(bound, 1e-30f));
        sc.hist[lane] = 0;
        sc.hist[lane + 32] = 0;
        const RangeSeq seq = range_seq(sz, cell.x, lane, sc.pref, sc.start);
        const int* order = G ? LV.order : nullptr;
        // pass 1: distances, kept for pass 2, and the bucket counts below the bound
        int pA = seq_index(seq, 32, lane, order);
        int pB = seq_index(seq, 0, lane, order);
        float4 vB = stream_point(pB, q, a.p4);
        for (int base = 0; base < seq.total; base += 32) {
            const int p = pB;
            const float4 v = vB;
            pB = pA;
            vB = stream_point(pB, q, a.p4);
            pA = seq_index(seq, base + 64, lane, order);
            float dd = 3.4e38f;
            if (p >= 0 && p != q) {
                dd = fs_dist3(pq.x, pq.y, pq.z, v.x, v.y, v.z);
                ++evals;
            }
            const int jj = base + lane;
            if (jj < kSelCache) sc.d[jj] = dd;
            if (dd < bound) atomicAdd(&sc.hist[sel_bucket(dd, scale)], 1);
        }
        __syncwarp();
        // the bucket of the (k+1)-th smallest below the bound
        const int h0 = sc.hist[2 * lane], h1 = sc.hist[2 * lane + 1];
        int incl = h0 + h1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int below = __shfl_sync(0xffffffffu, incl, 31);
        if (below < k + 1) continue;  // the block does not certify k+1 neighbours: next level
        const int excl = incl - h0 - h1;
        const int wl = __ffs(__ballot_sync(0xffffffffu, excl < k + 1 && incl >= k + 1)) - 1;
        int bstar = excl + h0 >= k + 1 ? 2 * lane : 2 * lane + 1;
        int cum = excl + h0 >= k + 1 ? excl + h0 : incl;
        bstar = __shfl_sync(0xffffffffu, bstar, wl);
        cum = __shfl_sync(0xffffffffu, cum, wl);
        gstart = G;
        if (cum > kSelCollect) return fail;  // too many candidates share the boundary bucket
        // pass 2: collect the candidates of buckets <= bstar
        int cnt = 0;
        const int cached = min(seq.total, kSelCache);
        for (int base = 0; base < cached; base += 32) {
            const int jj = base + lane;
            const float dd = jj < cached ? sc.d[jj] : 3.4e38f;
            const bool take = dd < bound && sel_bucket(dd, scale) <= bstar;
            const unsigned m = __ballot_sync(0xffffffffu, take);
            const int at = cnt + __popc(m & ((1u << lane) - 1u));
            if (take && at < kSelCollect) { sc.cd[at] = dd; sc.cj[at] = jj; }
            cnt += __popc(m);
        }
        if (seq.total > kSelCache) {  // recompute the distances beyond the kept ones
            for (int base = kSelCache; base < seq.total; base += 32) {
                const int p = seq_index(seq, base, lane, order);
                float dd = 3.4e38f;
                if (p >= 0 && p != q) {
                    const float4 v = __ldg(a.p4 + p);
                    dd = fs_dist3(pq.x, pq.y, pq.z, v.x, v.y, v.z);
                }
                const bool take = dd < bound && sel_bucket(dd, scale) <= bstar;
                const unsigned m = __ballot_sync(0xffffffffu, take);
                const int at = cnt + __popc(m & ((1u << lane) - 1u));
                if (take && at < kSelCollect) { sc.cd[at] = dd; sc.cj[at] = base + lane; }
                cnt += __popc(m);
            }
        }
        __syncwarp();
        if (cnt != cum) return fail;
        SelOut r = cnt <= 64 ? sel_finish<2>(a, np, q, pq, G, lane, sc, cnt, seq)
                             : sel_finish<4>(a, np, q, pq, G, lane, sc, cnt, seq);
        __syncwarp();  // the scratch is rewritten by the next query
        return r;
    }
    return fail;
}

}  // namespace
}  // namespace egt
