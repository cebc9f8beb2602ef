// Batched clouds: many independent point clouds through kNN -> EGT -> Taubin
// with one launch per stage (an extension of this project).
//
// Every cloud keeps the reference's per-cloud semantics: its own
// normalisation cube (GridKNNCuda.cu:1042-1071), its own 1024^3 cell grid and
// hierarchy, and its own k, so its lists, filtered lists and smoothed
// positions are those of a separate egt_create_cloud handle.  The clouds are
// slices of shared buffers:
//
//   points   [N]            cloud c = [off[c], off[c+1]), sorted by (c, key)
//   lists    [sum n_c*k_c]  cloud c at loff[c], row-major n_c x k_c
//   level L  order/cells    one sort over (c << 30 | level-L key); the cell
//                           tables of cloud c start at its first cell id plus
//                           c (one spare slot per cloud for the end sentinel)
//   rows     [count][B_L^2] per-cloud (y,z) row ranges, cloud-local cell ids
//
// A per-cloud descriptor (KnnArgs, built on the device) points into these
// slices, so the single-cloud search code runs unchanged.  The kNN is one
// persistent kernel whose warps claim chunks of queries of any cloud from one
// work counter.  The EGT filter is one warp-per-point kernel; its CSR has
// global column ids, so the Taubin loop runs over the union of the clouds'
// neighbourhoods with the single-cloud kernels (rows kept together per cloud
// by a cloud-major Morton order) as one captured graph.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "egt_filter.cuh"
#include "egt_internal.cuh"
#include "grid_common.cuh"
#include "knn_common.cuh"
#include "knn_search.cuh"
#include "knn_select.cuh"
#include "knn_tile.cuh"

using egt::KnnArgs;
using egt::LevelDev;
using egt::NormParams;
using egt::kMaxLevels;

struct egt_batch {
    egt_config cfg{};
    int count = 0;
    int64_t N = 0;
    int kmax = 0;
    int64_t lists_total = 0;
    std::vector<int64_t> off, loff;  // [count+1]
    std::vector<int> k;              // [count]
    egt_handle* h = nullptr;         // per-point buffers, stream, events, Taubin state (n = N)
    int64_t* d_off = nullptr;
    int64_t* d_loff = nullptr;
    int* d_k = nullptr;
    uint16_t* d_cloud = nullptr;     // [N] cloud of each point (same in input and sorted order)
    NormParams* d_np = nullptr;      // [count]
    unsigned long long* d_ctr = nullptr;  // [count][kCtrWords]
    int* order[kMaxLevels] = {};     // [N] levels >= 1, cloud-local indices
    int* cell_start[kMaxLevels] = {};  // [N + count + 1]
    int* cell_x[kMaxLevels] = {};
    int2* rows[kMaxLevels] = {};     // [count * B_L^2]
    int* cbase[kMaxLevels] = {};     // [count] first global cell id of each cloud
    KnnArgs* d_desc = nullptr;       // [count]
    int64_t* d_chunkoff = nullptr;   // [count+1] prefix of per-cloud query chunks
    int chunk = 0;                   // 0 = not tuned yet
    int chunkoff_for = 0;            // chunk size d_chunkoff was built for
    int taubin_mode = 0;
    int fuse = -1;                   // egt_batch_run: 1 fused kNN+EGT launch, 0 separate (-1: not tuned)
    float4* p4_input = nullptr;      // [N] sorted, normalised input positions (egt_batch_run starts here)
    bool tuning_fixed = false;
    bool have_knn = false, have_csr = false;
    egt_batch_timings tm{};
};

namespace egt {
namespace {

constexpr int kB = 256;  // threads per block of the per-point kernels

__global__ void k_cloud_ids(const int64_t* __restrict__ off, int count, int64_t N, uint16_t* __restrict__ cloud) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    int lo = 0, hi = count - 1;  // last c with off[c] <= i
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= i) lo = mid;
        else hi = mid - 1;
    }
    cloud[i] = (uint16_t)lo;
}

__global__ void k_init_extents_batch(uint32_t* acc, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count * 6) acc[i] = (i % 6) < 3 ? 0xffffffffu : 0u;
}

// Per-cloud per-axis min/max (warps inside one cloud reduce first).
__global__ void k_extents_batch(const float* __restrict__ xyz, int64_t N, const uint16_t* __restrict__ cloud,
                                uint32_t* __restrict__ acc) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool valid = i < N;
    const int c = valid ? cloud[i] : -1;
    float v[3] = {0.f, 0.f, 0.f};
    if (valid) {
        v[0] = xyz[3 * i];
        v[1] = xyz[3 * i + 1];
        v[2] = xyz[3 * i + 2];
    }
    const int c0 = __shfl_sync(0xffffffffu, c, 0);
    if (__all_sync(0xffffffffu, valid && c == c0)) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            float lo = v[d], hi = v[d];
            for (int o = 16; o > 0; o >>= 1) {
                lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
            }
            if ((threadIdx.x & 31) == 0) {
                atomicMin(&acc[6 * c + d], f2ord(lo));
                atomicMax(&acc[6 * c + 3 + d], f2ord(hi));
            }
        }
    } else if (valid) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            atomicMin(&acc[6 * c + d], f2ord(v[d]));
            atomicMax(&acc[6 * c + 3 + d], f2ord(v[d]));
        }
    }
}

__global__ void k_finalize_batch(const uint32_t* __restrict__ acc, float eps, float thres0,
                                 const int64_t* __restrict__ off, int count, NormParams* __restrict__ np) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= count) return;
    np[c] = finalize_norm(acc + 6 * c, eps, thres0, off[c + 1] - off[c]);
}

// normalize_points + level-0 key per cloud (same arithmetic as grid.cu), keyed
// above by the cloud id so that one stable sort orders every cloud.
__global__ void k_normalize_batch(const float* __restrict__ xyz, int64_t N, const uint16_t* __restrict__ cloud,
                                  const NormParams* __restrict__ nps, float4* __restrict__ tmp4,
                                  unsigned long long* __restrict__ key, int* __restrict__ idx) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int c = cloud[i];
    const NormParams p = nps[c];
    const float d = __fsub_rn(p.mx, p.mn);
    const float x = __fdiv_rn(__fsub_rn(xyz[3 * i], p.mn), d);
    const float y = __fdiv_rn(__fsub_rn(xyz[3 * i + 1], p.mn), d);
    const float z = __fdiv_rn(__fsub_rn(xyz[3 * i + 2], p.mn), d);
    tmp4[i] = make_float4(x, y, z, 0.f);
    const uint32_t xi = cell_coord(x, p.a, p.b, 1024), yi = cell_coord(y, p.a, p.b, 1024),
                   zi = cell_coord(z, p.a, p.b, 1024);
    key[i] = ((unsigned long long)c << 30) | (unsigned long long)(xi + yi * 1024u + zi * 1024u * 1024u);
    idx[i] = (int)i;
}

__global__ void k_gather_batch(const float4* __restrict__ tmp4, const int* __restrict__ sidx, int64_t N,
                               const uint16_t* __restrict__ cloud, const int64_t* __restrict__ off,
                               const NormParams* __restrict__ nps, float4* __restrict__ p4, float* __restrict__ x,
                               float* __restrict__ y, float* __restrict__ z, uint32_t* __restrict__ cell0,
                               int* __restrict__ perm) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= N) return;
    const int c = cloud[s];
    const NormParams p = nps[c];
    const int src = sidx[s];
    float4 v = tmp4[src];
    x[s] = v.x; y[s] = v.y; z[s] = v.z;
    const uint32_t xi = cell_coord(v.x, p.a, p.b, 1024), yi = cell_coord(v.y, p.a, p.b, 1024),
                   zi = cell_coord(v.z, p.a, p.b, 1024);
    const uint32_t packed = xi | (yi << 10) | (zi << 20);
    cell0[s] = packed;
    v.w = __uint_as_float(packed);
    p4[s] = v;
    perm[s] = (int)(src - off[c]);
}

__global__ void k_level_key_batch(const uint32_t* __restrict__ cell0, const uint16_t* __restrict__ cloud,
                                  const int64_t* __restrict__ off, int64_t N, int L,
                                  unsigned long long* __restrict__ key, int* __restrict__ val) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= N) return;
    const int c = cloud[s];
    const uint32_t cc = cell0[s], B = 1024u >> L;
    const uint32_t xi = (cc & 1023u) >> L, yi = ((cc >> 10) & 1023u) >> L, zi = ((cc >> 20) & 1023u) >> L;
    key[s] = ((unsigned long long)c << 30) | (unsigned long long)(xi + yi * B + zi * B * B);
    val[s] = (int)(s - off[c]);
}

__global__ void k_head_flags64(const unsigned long long* __restrict__ key, int64_t N, int* __restrict__ flag) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    flag[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}

// Per-cloud cell tables of one level (grid.cu k_cells per cloud slice).
__global__ void k_cells_batch(const unsigned long long* __restrict__ key, const int* __restrict__ flag,
                              const int* __restrict__ cid, const uint16_t* __restrict__ cloud,
                              const int64_t* __restrict__ off, int64_t N, int B, int L, int* __restrict__ cell_start,
                              int* __restrict__ cell_x, int2* __restrict__ rows, int* __restrict__ cbase,
                              unsigned long long* __restrict__ ctr) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int c = cloud[i];
    const int64_t o = off[c];
    const int nc_pts = (int)(off[c + 1] - o);
    const int cb = cid[o];
    const uint32_t UB = (uint32_t)B;
    const uint32_t mask = (1u << 30) - 1u;
    int2* rr = rows + (size_t)c * B * B;
    const uint32_t kk = (uint32_t)(key[i] & mask);
    if (i == o) cbase[c] = cb;
    if (i == o + nc_pts - 1) {
        const int nc = cid[i] + flag[i] - cb;
        cell_start[cb + c + nc] = nc_pts;
        rr[kk / UB].y = nc;
        ctr[(size_t)c * kCtrWords + kCtrNcells + L] = (unsigned long long)nc;
    }
    if (!flag[i]) return;
    const int lc = cid[i] - cb;
    const int slot = cid[i] + c;
    cell_start[slot] = (int)(i - o);
    cell_x[slot] = (int)(kk % UB);
    const uint32_t row = kk / UB;
    if (lc == 0) {
        rr[row].x = 0;
    } else {
        const uint32_t prow = (uint32_t)(key[i - 1] & mask) / UB;
        if (prow != row) {
            rr[prow].y = lc;
            rr[row].x = lc;
        }
    }
}

struct DescArgs {
    const float4* p4;
    const NormParams* np;
    int* order[kMaxLevels];
    int* cell_start[kMaxLevels];
    int* cell_x[kMaxLevels];
    int2* rows[kMaxLevels];
    const int* cbase[kMaxLevels];
    const int64_t* off;
    const int64_t* loff;
    const int* k;
    int count, max_pts, chunk;
    int* lists;
    float* kth;
    uint8_t* qlevel;
    unsigned long long* ctr;
};

__global__ void k_make_desc(DescArgs d, KnnArgs* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.count) return;
    const int64_t o = d.off[c];
    KnnArgs a;
    a.p4 = d.p4 + o;
    a.np = d.np + c;
    for (int L = 0; L < kMaxLevels; L++) {
        const int B = 1024 >> L;
        const int cb = d.cbase[L][c];
        a.lv[L].B = B;
        a.lv[L].ncells = (int)d.ctr[(size_t)c * kCtrWords + kCtrNcells + L];
        a.lv[L].order = L == 0 ? nullptr : d.order[L] + o;
        a.lv[L].cell_start = d.cell_start[L] + cb + c;
        a.lv[L].cell_x = d.cell_x[L] + cb + c;
        a.lv[L].row_range = d.rows[L] + (size_t)c * B * B;
    }
    a.n = (int)(d.off[c + 1] - o);
    a.k = d.k[c];
    a.max_pts = d.max_pts;
    a.chunk = d.chunk;
    a.lists = d.lists + d.loff[c];
    a.kth_out = d.kth + o;
    a.qlevel = d.qlevel + o;
    a.counters = d.ctr + (size_t)c * kCtrWords;
    a.gbase = o;
    out[c] = a;
}

__global__ void k_set_chunk(KnnArgs* __restrict__ desc, int count, int chunk) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < count) desc[c].chunk = chunk;
}

// Persistent kNN over all clouds: a warp claims one chunk of queries of some
// cloud per atomic (chunks of cloud c are [chunkoff[c], chunkoff[c+1])).
template <int S>
__global__ void __launch_bounds__(kWarps * 32) k_knn_batch(const KnnArgs* __restrict__ desc,
                                                           const int64_t* __restrict__ chunkoff, int count,
                                                           unsigned long long* __restrict__ work) {
    __shared__ int s_pref[kWarps][32];
    __shared__ int s_start[kWarps][32];
    __shared__ float s_md[kWarps][32 * S];
    __shared__ int s_mp[kWarps][32 * S];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t total = chunkoff[count];
    for (;;) {
        unsigned long long g = 0;
        if (lane == 0) g = atomicAdd(work, 1ull);
        g = __shfl_sync(0xffffffffu, g, 0);
        if ((int64_t)g >= total) break;
        int lo = 0, hi = count - 1;  // cloud of chunk g
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (chunkoff[mid] <= (int64_t)g) lo = mid;
            else hi = mid - 1;
        }
        const KnnArgs& a = desc[lo];
        const NormParams np = *a.np;
        const int q0 = (int)(((int64_t)g - chunkoff[lo]) * a.chunk);
        const int q1 = min(q0 + a.chunk, a.n);
        for (int q = q0; q < q1; q++) {
            WarpList<S> L;
            bool invalid, rerun;
            const int reached = plain_query<true, S>(a, np, q, a.p4[q], L, invalid, lane, s_pref[w], s_start[w],
                                                     s_md[w], s_mp[w], rerun);
            write_query<S>(a, q, L, invalid, reached, lane);
            if (rerun && lane == 0) atomicAdd(&a.counters[kCtrExactRerun], 1ull);
        }
    }
}

// kNN and EGT filter of every cloud in one persistent launch: a warp claims
// one chunk of queries of some cloud per atomic, runs the reference's ring
// search for each query (as k_knn_batch does), then filters the query's list
// with the EGT test (egt_query, one query per warp) and stores its kept count
// for the CSR.  S: list registers for k+1 slots; Se: filter slots per lane.
template <int S, int Se>
__global__ void __launch_bounds__(kWarps * 32, 3) k_knn_egt_batch(const KnnArgs* __restrict__ desc,
                                                                  const int64_t* __restrict__ chunkoff, int count,
                                                                  unsigned long long* __restrict__ work, float alpha,
                                                                  int* __restrict__ counts) {
    __shared__ SelScratch s_sc[kWarps];  // ring-search scratch, then the filter's staged positions
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    SelScratch& sc = s_sc[w];
    const int64_t total = chunkoff[count];
    for (;;) {
        unsigned long long g = 0;
        if (lane == 0) g = atomicAdd(work, 1ull);
        g = __shfl_sync(0xffffffffu, g, 0);
        if ((int64_t)g >= total) break;
        int lo = 0, hi = count - 1;  // cloud of chunk g
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (chunkoff[mid] <= (int64_t)g) lo = mid;
            else hi = mid - 1;
        }
        const KnnArgs& a = desc[lo];
        const NormParams np = *a.np;
        const int q0 = (int)(((int64_t)g - chunkoff[lo]) * a.chunk);
        const int q1 = min(q0 + a.chunk, a.n);
        for (int q = q0; q < q1; q++) {
            const float4 pq = a.p4[q];
            WarpList<S> L;
            bool invalid, rerun;
            const int reached = plain_query<true, S>(a, np, q, pq, L, invalid, lane, sc.pref, sc.start, sc.cd, sc.cj,
                                                     rerun);
            write_query<S>(a, q, L, invalid, reached, lane);
            if (rerun && lane == 0) atomicAdd(&a.counters[kCtrExactRerun], 1ull);
            __syncwarp();  // the row is written; the scratch is reused
            unsigned tests = 0;  // not reported for batches
            const int cnt = egt_query<Se, 32>(a.p4, pq, a.lists + (size_t)q * a.k, a.k, alpha, lane, tests,
                                              reinterpret_cast<float4*>(sc.d));
            if (lane == 0) counts[a.gbase + q] = cnt;
            __syncwarp();
        }
    }
}

// Largest k the fused launch takes (k+1 list slots in three registers per lane).
constexpr int kFusedMaxK = 95;

// One query per group of G lanes (32 / G queries per warp, possibly of
// different clouds: each group filters with its own cloud's k).
template <int S, int G>
__global__ void __launch_bounds__(kWarps * 32, S <= 3 ? 4 : 1) k_egt_batch(
    const float4* __restrict__ p4, int* __restrict__ lists, const uint16_t* __restrict__ cloud,
    const int64_t* __restrict__ off, const int64_t* __restrict__ loff, const int* __restrict__ kk, int64_t N,
    float alpha, int* __restrict__ counts) {
    constexpr int kPer = 32 / G;
    __shared__ float4 s_v[kWarps * kPer][G * S];
    const int lane = threadIdx.x & 31;
    const int64_t i0 = (blockIdx.x * (int64_t)kWarps + (threadIdx.x >> 5)) * kPer;
    if (i0 >= N) return;  // whole warps only
    const int64_t i = i0 + lane / G;
    const bool active = i < N;
    const int c = active ? cloud[i] : 0;
    const int64_t o = off[c];
    const int k = kk[c];
    unsigned tests = 0;  // not reported for batches
    const int cnt = egt_query<S, G>(p4 + o, active ? p4[i] : make_float4(0.f, 0.f, 0.f, 0.f),
                                    lists + loff[c] + (active ? i - o : 0) * k, k, alpha, lane, tests,
                                    s_v[(threadIdx.x >> 5) * kPer + lane / G], active);
    if (active && (lane & (G - 1)) == 0) counts[i] = cnt;
}

__global__ void k_count_batch(const int* __restrict__ lists, const uint16_t* __restrict__ cloud,
                              const int64_t* __restrict__ off, const int64_t* __restrict__ loff,
                              const int* __restrict__ kk, int64_t N, int* __restrict__ counts) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int c = cloud[i];
    const int k = kk[c];
    const int* row = lists + loff[c] + (i - off[c]) * k;
    int n = 0;
    for (int j = 0; j < k; j++) n += row[j] >= 0;
    counts[i] = n;
}

// Kept entries of every row, in list order, as global column ids.
template <int S>
__global__ void __launch_bounds__(kWarps * 32) k_compact_batch(const int* __restrict__ lists,
                                                               const uint16_t* __restrict__ cloud,
                                                               const int64_t* __restrict__ off,
                                                               const int64_t* __restrict__ loff,
                                                               const int* __restrict__ kk, int64_t N,
                                                               const int* __restrict__ csr_off,
                                                               int* __restrict__ col) {
    const int lane = threadIdx.x & 31;
    const int64_t i = blockIdx.x * (int64_t)kWarps + (threadIdx.x >> 5);
    if (i >= N) return;
    const int c = cloud[i];
    const int64_t o = off[c];
    const int k = kk[c];
    const int* row = lists + loff[c] + (i - o) * k;
    int base = csr_off[i];
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        const int v = t < k ? row[t] : -1;
        const unsigned m = __ballot_sync(0xffffffffu, v >= 0);
        if (v >= 0) col[base + __popc(m & ((1u << lane) - 1u))] = (int)(v + o);
        base += __popc(m);
    }
}

__global__ void k_output_batch(const float4* __restrict__ p4, const int* __restrict__ perm,
                               const uint16_t* __restrict__ cloud, const int64_t* __restrict__ off,
                               const NormParams* __restrict__ nps, int64_t N, float* __restrict__ out) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= N) return;
    const int c = cloud[s];
    const float mn = nps[c].mn, d = __fsub_rn(nps[c].mx, nps[c].mn);
    const float4 v = p4[s];
    const int64_t o = off[c] + perm[s];
    out[3 * o] = __fmaf_rn(v.x, d, mn);
    out[3 * o + 1] = __fmaf_rn(v.y, d, mn);
    out[3 * o + 2] = __fmaf_rn(v.z, d, mn);
}

__global__ void k_lists_cloud(const int* __restrict__ lists, const int* __restrict__ perm, int n, int k,
                              int* __restrict__ out) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * k) return;
    const int s = (int)(e / k), j = (int)(e % k);
    const int v = lists[e];
    out[(size_t)perm[s] * k + j] = v >= 0 ? perm[v] : -1;
}

unsigned blocks(int64_t n, int per = kB) { return (unsigned)((n + per - 1) / per); }

template <int S, int G>
egt_status launch_egt_batch(egt_batch* b, float alpha, int* counts, cudaStream_t st) {
    k_egt_batch<S, G><<<blocks(b->N, kWarps * (32 / G)), kWarps * 32, 0, st>>>(
        b->h->p4, b->h->lists, b->d_cloud, b->d_off, b->d_loff, b->d_k, b->N, alpha, counts);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

template <int S>
egt_status launch_compact_batch(egt_batch* b, cudaStream_t st) {
    k_compact_batch<S><<<blocks(b->N, kWarps), kWarps * 32, 0, st>>>(
        b->h->lists, b->d_cloud, b->d_off, b->d_loff, b->d_k, b->N, b->h->csr_off, b->h->csr_col);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

// Blocks of one resident wave of k_knn_batch<S>.
// Largest cell population of each cloud and level (the cell-tile search's
// oversized-cell check): block (cloud, level).
__global__ void __launch_bounds__(256) k_maxpop_batch(const KnnArgs* __restrict__ desc) {
    const KnnArgs& a = desc[blockIdx.x];
    const LevelDev& LV = a.lv[blockIdx.y];
    int v = 0;
    for (int i = threadIdx.x; i < LV.ncells; i += blockDim.x) v = max(v, LV.cell_start[i + 1] - LV.cell_start[i]);
    v = __reduce_max_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0 && v > 0) atomicMax(&a.counters[kCtrMaxPop + blockIdx.y], (unsigned long long)v);
}

// The ring search of the queries in `list` (indices over all clouds' points),
// one query per warp.
template <int S>
__global__ void __launch_bounds__(kWarps * 32) k_knn_list_batch(const KnnArgs* __restrict__ desc,
                                                                const uint16_t* __restrict__ cloud,
                                                                const int* __restrict__ list,
                                                                const unsigned long long* __restrict__ n_list,
                                                                unsigned long long* __restrict__ work) {
    __shared__ int s_pref[kWarps][32];
    __shared__ int s_start[kWarps][32];
    __shared__ float s_md[kWarps][32 * S];
    __shared__ int s_mp[kWarps][32 * S];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned long long n = *n_list;
    for (;;) {
        unsigned long long j = 0;
        if (lane == 0) j = atomicAdd(work, 1ull);
        j = __shfl_sync(0xffffffffu, j, 0);
        if (j >= n) break;
        const int i = list[j];
        const KnnArgs& a = desc[cloud[i]];
        const int q = i - (int)a.gbase;
        const NormParams np = *a.np;
        WarpList<S> L;
        bool invalid, rerun;
        const int reached = plain_query<true, S>(a, np, q, a.p4[q], L, invalid, lane, s_pref[w], s_start[w], s_md[w],
                                                 s_mp[w], rerun);
        write_query<S>(a, q, L, invalid, reached, lane);
        if (rerun && lane == 0) atomicAdd(&a.counters[kCtrExactRerun], 1ull);
    }
}

template <int S>
egt_status knn_wave(int device, unsigned* out) {
    static std::mutex mu;
    static std::map<int, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(device);
    if (it == cache.end()) {
        int sms = 0, per = 0;
        EGT_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        EGT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_knn_batch<S>, kWarps * 32, 0));
        it = cache.emplace(device, std::max(1, sms * std::max(per, 1))).first;
    }
    *out = (unsigned)it->second;
    return EGT_OK;
}

template <int S>
egt_status run_knn_batch_s(egt_batch* b, cudaStream_t st) {
    unsigned G = 0;
    EGT_TRY(knn_wave<S>(b->cfg.device, &G));
    k_knn_batch<S><<<G, kWarps * 32, 0, st>>>(b->d_desc, b->d_chunkoff, b->count, b->h->d_counters + kCtrWork);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

// Blocks of one resident wave of a kernel, per (kernel, device).
template <typename K>
egt_status kernel_wave(K kernel, int device, unsigned* out) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), device);
    auto it = cache.find(key);
    if (it == cache.end()) {
        int sms = 0, per = 0;
        EGT_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        EGT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kWarps * 32, 0));
        it = cache.emplace(key, std::max(1, sms * std::max(per, 1))).first;
    }
    *out = (unsigned)it->second;
    return EGT_OK;
}

template <int S, int Se>
egt_status run_knn_egt_batch_s(egt_batch* b, float alpha, int* counts, cudaStream_t st) {
    unsigned G = 0;
    EGT_TRY(kernel_wave(k_knn_egt_batch<S, Se>, b->cfg.device, &G));
    k_knn_egt_batch<S, Se><<<G, kWarps * 32, 0, st>>>(b->d_desc, b->d_chunkoff, b->count,
                                                      b->h->d_counters + kCtrWork, alpha, counts);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

// (Re)builds the chunk prefix and the descriptors' chunk for `chunk`.
egt_status set_chunk(egt_batch* b, int chunk) {
    if (b->chunkoff_for == chunk) return EGT_OK;
    std::vector<int64_t> co(b->count + 1, 0);
    for (int c = 0; c < b->count; c++) co[c + 1] = co[c] + (b->off[c + 1] - b->off[c] + chunk - 1) / chunk;
    cudaStream_t st = b->h->stream;
    EGT_CUDA_TRY(cudaMemcpyAsync(b->d_chunkoff, co.data(), sizeof(int64_t) * (b->count + 1), cudaMemcpyHostToDevice, st));
    k_set_chunk<<<blocks(b->count), kB, 0, st>>>(b->d_desc, b->count, chunk);
    EGT_LAUNCH_CHECK();
    EGT_CUDA_TRY(cudaStreamSynchronize(st));  // `co` is pageable host memory
    b->chunkoff_for = chunk;
    return EGT_OK;
}

// The cell-tile search over every cloud (clouds whose k lies outside
// [kTileMinK, kTileMaxK] run the ring search), then the ring search of the
// queries it could not certify.
template <int S>
egt_status knn_batch_tile(egt_batch* b, cudaStream_t st) {
    TileArgs t;
    EGT_TRY(tile_prepare(b->h, &t));
    t.desc = b->d_desc;
    t.cloud_of = b->d_cloud;
    t.npts = (int)b->N;
    EGT_CUDA_TRY(cudaMemset2DAsync(b->d_ctr + kCtrMaxPop, sizeof(unsigned long long) * kCtrWords, 0,
                                   kMaxLevels * sizeof(unsigned long long), b->count, st));
    k_maxpop_batch<<<dim3(b->count, kMaxLevels), 256, 0, st>>>(b->d_desc);
    EGT_LAUNCH_CHECK();
    int kt = 0;  // the largest k the tile search takes
    for (int c = 0; c < b->count; c++)
        if (b->k[c] >= kTileMinK && b->k[c] <= kTileMaxK) kt = std::max(kt, b->k[c]);
    KnnArgs none{};  // each cloud's arguments come from its descriptor
    EGT_TRY(tile_launch<true>(none, t, kt, st));
    unsigned G = 0;
    EGT_TRY(kernel_wave(k_knn_list_batch<S>, b->cfg.device, &G));
    k_knn_list_batch<S><<<G, kWarps * 32, 0, st>>>(b->d_desc, b->d_cloud, t.ring2, t.n_ring2,
                                                   b->h->d_counters + kCtrTileRingWork);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

egt_status knn_batch(egt_batch* b) {
    cudaStream_t st = b->h->stream;
    EGT_TRY(set_chunk(b, b->chunk > 0 ? b->chunk : kChunk));
    // reset every cloud's kNN counters and the shared work counter
    EGT_CUDA_TRY(cudaMemsetAsync(b->h->d_counters + kCtrWork, 0, sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaMemset2DAsync(b->d_ctr + kCtrInvalid, sizeof(unsigned long long) * kCtrWords, 0,
                                   2 * sizeof(unsigned long long), b->count, st));
    EGT_CUDA_TRY(cudaMemset2DAsync(b->d_ctr + kCtrExactRerun, sizeof(unsigned long long) * kCtrWords, 0,
                                   sizeof(unsigned long long), b->count, st));
    EGT_CUDA_TRY(cudaEventRecord(b->h->ev[2], st));
    const int kk = b->kmax;
    bool tile = b->cfg.knn_mode == EGT_KNN_TILE;
    if (tile) {
        tile = false;
        for (int c = 0; c < b->count; c++) tile |= b->k[c] >= kTileMinK && b->k[c] <= kTileMaxK;
    }
    if (tile) {
        if (kk + 1 <= 32) EGT_TRY(knn_batch_tile<1>(b, st));
        else if (kk + 1 <= 64) EGT_TRY(knn_batch_tile<2>(b, st));
        else if (kk + 1 <= 96) EGT_TRY(knn_batch_tile<3>(b, st));
        else if (kk + 1 <= 128) EGT_TRY(knn_batch_tile<4>(b, st));
        else EGT_TRY(knn_batch_tile<8>(b, st));
    } else if (kk + 1 <= 32) EGT_TRY(run_knn_batch_s<1>(b, st));
    else if (kk + 1 <= 64) EGT_TRY(run_knn_batch_s<2>(b, st));
    else if (kk + 1 <= 96) EGT_TRY(run_knn_batch_s<3>(b, st));
    else if (kk + 1 <= 128) EGT_TRY(run_knn_batch_s<4>(b, st));
    else EGT_TRY(run_knn_batch_s<8>(b, st));
    EGT_CUDA_TRY(cudaEventRecord(b->h->ev[3], st));
    b->have_knn = true;
    b->have_csr = false;
    b->h->have_csr = false;
    return EGT_OK;
}

// CSR of the current lists (after the filter or unfiltered).
egt_status csr_batch(egt_batch* b, int* counts) {
    cudaStream_t st = b->h->stream;
    egt_handle* h = b->h;
    const int64_t N = b->N;
    size_t t_scan = 0;
    EGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, t_scan, (int*)nullptr, (int*)nullptr, (int)(N + 1), st));
    void* tmp = nullptr;
    EGT_TRY(scratch_reserve(h, t_scan, &tmp));
    if (!h->csr_off) EGT_CUDA_TRY(dev_alloc(h, &h->csr_off, sizeof(int) * (N + 1)));
    if (!h->csr_col) {
        EGT_CUDA_TRY(dev_alloc(h, &h->csr_col, sizeof(int) * std::max<int64_t>(b->lists_total, 1)));
        h->csr_cap = std::max<int64_t>(b->lists_total, 1);
    }
    EGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, t_scan, counts, h->csr_off, (int)(N + 1), st));
    const int kk = b->kmax;
    if (kk <= 32) EGT_TRY(launch_compact_batch<1>(b, st));
    else if (kk <= 64) EGT_TRY(launch_compact_batch<2>(b, st));
    else if (kk <= 128) EGT_TRY(launch_compact_batch<4>(b, st));
    else EGT_TRY(launch_compact_batch<8>(b, st));
    h->nnz = -1;
    h->have_csr = true;
    h->csr_version++;
    b->have_csr = true;
    return EGT_OK;
}

egt_status filter_batch(egt_batch* b, float alpha) {
    cudaStream_t st = b->h->stream;
    const int64_t N = b->N;
    int* counts = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&counts, sizeof(int) * (N + 1), st));
    EGT_CUDA_TRY(cudaMemsetAsync(counts + N, 0, sizeof(int), st));
    EGT_CUDA_TRY(cudaEventRecord(b->h->ev[4], st));
    const int kk = b->kmax;
    egt_status s;
    // lanes per query as in the single-cloud filter, from the largest k of the batch
    if (kk <= 16) s = launch_egt_batch<1, 16>(b, alpha, counts, st);
    else if (kk <= 32) s = launch_egt_batch<1, 32>(b, alpha, counts, st);
    else if (kk <= 48) s = launch_egt_batch<3, 16>(b, alpha, counts, st);
    else if (kk <= 64) s = launch_egt_batch<2, 32>(b, alpha, counts, st);
    else if (kk <= 128) s = launch_egt_batch<4, 32>(b, alpha, counts, st);
    else s = launch_egt_batch<8, 32>(b, alpha, counts, st);
    if (s == EGT_OK) s = csr_batch(b, counts);
    EGT_CUDA_TRY(cudaEventRecord(b->h->ev[5], st));
    cudaFreeAsync(counts, st);
    return s;
}

// kNN and EGT filter of every cloud in one persistent launch (the lists end
// filtered), then the CSR of the kept neighbours.  knn_ms times the fused
// launch, egt_ms the CSR packing.
egt_status knn_egt_batch(egt_batch* b, float alpha) {
    cudaStream_t st = b->h->stream;
    const int64_t N = b->N;
    EGT_TRY(set_chunk(b, b->chunk > 0 ? b->chunk : kChunk));
    EGT_CUDA_TRY(cudaMemsetAsync(b->h->d_counters + kCtrWork, 0, sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaMemset2DAsync(b->d_ctr + kCtrInvalid, sizeof(unsigned long long) * kCtrWords, 0,
                                   2 * sizeof(unsigned long long), b->count, st));
    EGT_CUDA_TRY(cudaMemset2DAsync(b->d_ctr + kCtrExactRerun, sizeof(unsigned long long) * kCtrWords, 0,
                                   sizeof(unsigned long long), b->count, st));
    int* counts = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&counts, sizeof(int) * (N + 1), st));
    EGT_CUDA_TRY(cudaMemsetAsync(counts + N, 0, sizeof(int), st));
    EGT_CUDA_TRY(cudaEventRecord(b->h->ev[2], st));
    const int kk = b->kmax;
    egt_status s = kk + 1 <= 32   ? run_knn_egt_batch_s<1, 1>(b, alpha, counts, st)
                   : kk + 1 <= 64 ? run_knn_egt_batch_s<2, 2>(b, alpha, counts, st)
                                  : run_knn_egt_batch_s<3, 3>(b, alpha, counts, st);
    if (s == EGT_OK) s = cudaEventRecord(b->h->ev[3], st) == cudaSuccess ? EGT_OK : EGT_ERR_CUDA;
    if (s == EGT_OK) s = cudaEventRecord(b->h->ev[4], st) == cudaSuccess ? EGT_OK : EGT_ERR_CUDA;
    b->have_knn = true;
    if (s == EGT_OK) s = csr_batch(b, counts);
    if (s == EGT_OK) s = cudaEventRecord(b->h->ev[5], st) == cudaSuccess ? EGT_OK : EGT_ERR_CUDA;
    cudaFreeAsync(counts, st);
    b->tm.fused = s == EGT_OK ? 1 : 0;
    return s;
}

egt_status ensure_csr_batch(egt_batch* b) {
    if (b->have_csr) return EGT_OK;
    cudaStream_t st = b->h->stream;
    const int64_t N = b->N;
    int* counts = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&counts, sizeof(int) * (N + 1), st));
    EGT_CUDA_TRY(cudaMemsetAsync(counts + N, 0, sizeof(int), st));
    k_count_batch<<<blocks(N), kB, 0, st>>>(b->h->lists, b->d_cloud, b->d_off, b->d_loff, b->d_k, N, counts);
    EGT_LAUNCH_CHECK();
    egt_status s = csr_batch(b, counts);
    cudaFreeAsync(counts, st);
    return s;
}

egt_status taubin_batch(egt_batch* b, int iters, float lambda, float mu) {
    EGT_TRY(ensure_csr_batch(b));
    b->h->taubin_mode = b->taubin_mode;
    return run_taubin(b->h, iters, lambda, mu);
}

// Autotuner: times each kNN work chunk and each Taubin half-step kernel on the
// batch itself; results are cached per (log2 points, max k) bucket.
struct TuneKey {
    int device, logn, kmax;
    bool operator<(const TuneKey& o) const {
        return std::tie(device, logn, kmax) < std::tie(o.device, o.logn, o.kmax);
    }
};
std::mutex g_tune_mu;
struct TuneVal {
    int chunk, taubin_mode, fuse;
};
std::map<TuneKey, TuneVal> g_tune;

egt_status autotune(egt_batch* b, float lambda, float mu, float alpha) {
    if (b->tuning_fixed || b->chunk > 0) return EGT_OK;
    const TuneKey key{b->cfg.device, (int)std::lround(std::log2((double)b->N)), b->kmax};
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            b->chunk = it->second.chunk;
            b->taubin_mode = it->second.taubin_mode;
            b->fuse = it->second.fuse;
            return EGT_OK;
        }
    }
    egt_handle* h = b->h;
    cudaStream_t st = h->stream;
    cudaEvent_t t0, t1;
    EGT_CUDA_TRY(cudaEventCreate(&t0));
    EGT_CUDA_TRY(cudaEventCreate(&t1));
    EGT_CUDA_TRY(cudaEventRecord(t0, st));
    float best = 1e30f;
    int best_chunk = kChunk;
    b->chunk = kChunk;
    EGT_TRY(knn_batch(b));  // warm
    for (int c : {1, 2, 4, 8, 16}) {
        b->chunk = c;
        EGT_TRY(knn_batch(b));
        EGT_CUDA_TRY(cudaEventSynchronize(h->ev[3]));
        const float ms = elapsed_ms(h->ev[2], h->ev[3]);
        if (ms < best) { best = ms; best_chunk = c; }
    }
    b->chunk = best_chunk;
    // kNN + filter: one fused launch or two, whichever is faster here
    b->fuse = 0;
    bool filtered = false;  // the lists are filtered and the CSR built (by the two-launch run)
    if (b->kmax <= kFusedMaxK) {
        EGT_TRY(knn_egt_batch(b, alpha));  // warm
        EGT_TRY(knn_egt_batch(b, alpha));
        EGT_CUDA_TRY(cudaEventSynchronize(h->ev[5]));
        const float fused_ms = elapsed_ms(h->ev[2], h->ev[5]);
        EGT_TRY(knn_batch(b));
        EGT_TRY(filter_batch(b, alpha));
        EGT_CUDA_TRY(cudaEventSynchronize(h->ev[5]));
        const float sep_ms = elapsed_ms(h->ev[2], h->ev[3]) + elapsed_ms(h->ev[4], h->ev[5]);
        b->fuse = fused_ms < sep_ms ? 1 : 0;
        b->tm.fused_ms = fused_ms;
        b->tm.separate_ms = sep_ms;
        filtered = true;
    }
    // Taubin kernel: a few half-steps of each on a copy of the positions
    if (!filtered) EGT_TRY(filter_batch(b, alpha));
    float4* save = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&save, sizeof(float4) * b->N, st));
    EGT_CUDA_TRY(cudaMemcpyAsync(save, h->p4, sizeof(float4) * b->N, cudaMemcpyDeviceToDevice, st));
    float tbest = 1e30f;
    int best_mode = 0;
    for (int mode : {0, 1}) {
        b->taubin_mode = mode;
        EGT_TRY(taubin_batch(b, 10, lambda, mu));  // capture + warm
        EGT_TRY(taubin_batch(b, 10, lambda, mu));
        EGT_CUDA_TRY(cudaEventSynchronize(h->ev[7]));
        const float ms = elapsed_ms(h->ev[6], h->ev[7]);
        if (ms < tbest) { tbest = ms; best_mode = mode; }
        EGT_CUDA_TRY(cudaMemcpyAsync(h->p4, save, sizeof(float4) * b->N, cudaMemcpyDeviceToDevice, st));
    }
    cudaFreeAsync(save, st);
    b->taubin_mode = best_mode;
    b->have_csr = false;  // the filter runs again in the measured pipeline
    h->have_csr = false;
    EGT_CUDA_TRY(cudaEventRecord(t1, st));
    EGT_CUDA_TRY(cudaEventSynchronize(t1));
    b->tm.tune_ms = elapsed_ms(t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = {b->chunk, b->taubin_mode, b->fuse};
    return EGT_OK;
}

void free_batch(egt_batch* b) {
    if (!b) return;
    if (b->h) {
        egt_handle* h = b->h;
        auto F = [h](void* p) { dev_free(h, p); };
        F(b->d_off); F(b->d_loff); F(b->d_k); F(b->d_cloud); F(b->d_np); F(b->d_ctr); F(b->d_desc);
        F(b->d_chunkoff); F(b->p4_input);
        for (int L = 0; L < kMaxLevels; L++) {
            F(b->order[L]); F(b->cell_start[L]); F(b->cell_x[L]); F(b->rows[L]); F(b->cbase[L]);
        }
        // lists/kth/qlevel/CSR/Taubin buffers belong to the handle
        delete_handle(h);
    }
    delete b;
}

}  // namespace
}  // namespace egt

using namespace egt;

extern "C" {

egt_status egt_batch_create(const float* xyz_host, const int64_t* offsets, const int* k, int count,
                            const egt_config* cfg_in, void* stream, egt_batch** out) {
    if (!out) { set_error("egt_batch_create: null output"); return EGT_ERR_ARG; }
    *out = nullptr;
    if (!xyz_host || !offsets || !k || count < 1 || count > 65535) {
        set_error("egt_batch_create: bad argument (count in [1, 65535])");
        return EGT_ERR_ARG;
    }
    if (offsets[0] != 0) { set_error("egt_batch_create: offsets[0] must be 0"); return EGT_ERR_ARG; }
    int64_t lists_total = 0;
    int kmax = 0;
    for (int c = 0; c < count; c++) {
        const int64_t n = offsets[c + 1] - offsets[c];
        if (n < 1 || n > (int64_t)(1u << 30)) { set_error("egt_batch_create: every cloud needs 1..2^30 points"); return EGT_ERR_ARG; }
        if (k[c] < 1 || k[c] > 255) { set_error("egt_batch_create: k must be in [1, 255]"); return EGT_ERR_ARG; }
        lists_total += n * k[c];
        kmax = std::max(kmax, k[c]);
    }
    const int64_t N = offsets[count];
    if (N > (int64_t)(1u << 30) || lists_total > (int64_t)0x7fffffff) {
        set_error("egt_batch_create: total points must be <= 2^30 and total list entries < 2^31");
        return EGT_ERR_ARG;
    }
    egt_config cfg;
    egt_default_config(&cfg);
    if (cfg_in) cfg = *cfg_in;
    if (cfg.bucket_count != 1024) { set_error("bucket_count must be 1024 (the reference's level-0 grid)"); return EGT_ERR_ARG; }
    if (cfg.max_points_in_cell < 1) { set_error("max_points_in_cell must be >= 1"); return EGT_ERR_ARG; }
    egt_batch* b = new egt_batch();
    b->cfg = cfg;
    b->count = count;
    b->N = N;
    b->kmax = kmax;
    b->lists_total = lists_total;
    b->off.assign(offsets, offsets + count + 1);
    b->k.assign(k, k + count);
    b->loff.assign(count + 1, 0);
    for (int c = 0; c < count; c++) b->loff[c + 1] = b->loff[c] + (offsets[c + 1] - offsets[c]) * k[c];
    egt_status s = new_bare_handle(cfg, N, (cudaStream_t)stream, &b->h);
    if (s != EGT_OK) { delete b; return s; }
    egt_handle* h = b->h;
    cudaStream_t st = h->stream;
    auto fail = [&](egt_status e) { free_batch(b); return e; };
#define BTRY(call)                                                                             \
    do {                                                                                       \
        cudaError_t e__ = (call);                                                              \
        if (e__ != cudaSuccess) {                                                              \
            set_error(cuda_msg(e__, #call, __FILE__, __LINE__));                               \
            return fail(e__ == cudaErrorMemoryAllocation ? EGT_ERR_NOMEM : EGT_ERR_CUDA);      \
        }                                                                                      \
    } while (0)
#define BSTAT(call)                      \
    do {                                 \
        egt_status s__ = (call);         \
        if (s__ != EGT_OK) return fail(s__); \
    } while (0)
    int bits = 0;
    while ((1 << bits) < count) bits++;
    h->cloud_bits = bits;
    BTRY(dev_alloc(h, &b->d_off, sizeof(int64_t) * (count + 1)));
    BTRY(dev_alloc(h, &b->d_loff, sizeof(int64_t) * (count + 1)));
    BTRY(dev_alloc(h, &b->d_k, sizeof(int) * count));
    BTRY(dev_alloc(h, &b->d_cloud, sizeof(uint16_t) * N));
    BTRY(dev_alloc(h, &b->d_np, sizeof(NormParams) * count));
    BTRY(dev_alloc(h, &b->d_ctr, sizeof(unsigned long long) * kCtrWords * count));
    BTRY(dev_alloc(h, &b->d_desc, sizeof(KnnArgs) * count));
    BTRY(dev_alloc(h, &b->d_chunkoff, sizeof(int64_t) * (count + 1)));
    BTRY(dev_alloc(h, &h->lists, sizeof(int) * lists_total));
    BTRY(dev_alloc(h, &h->kth, sizeof(float) * N));
    BTRY(dev_alloc(h, &h->qlevel, N));
    h->k = kmax;
    h->cloud_of = b->d_cloud;
    BTRY(cudaMemcpyAsync(b->d_off, b->off.data(), sizeof(int64_t) * (count + 1), cudaMemcpyHostToDevice, st));
    BTRY(cudaMemcpyAsync(b->d_loff, b->loff.data(), sizeof(int64_t) * (count + 1), cudaMemcpyHostToDevice, st));
    BTRY(cudaMemcpyAsync(b->d_k, b->k.data(), sizeof(int) * count, cudaMemcpyHostToDevice, st));
    BTRY(cudaMemsetAsync(b->d_ctr, 0, sizeof(unsigned long long) * kCtrWords * count, st));
    // points to the device
    float* dxyz = nullptr;
    BTRY(cudaMallocAsync((void**)&dxyz, sizeof(float) * 3 * N, st));
    BTRY(cudaMemcpyAsync(dxyz, xyz_host, sizeof(float) * 3 * N, cudaMemcpyHostToDevice, st));
    BTRY(cudaEventRecord(h->ev[0], st));
    k_cloud_ids<<<blocks(N), kB, 0, st>>>(b->d_off, count, N, b->d_cloud);
    BSTAT([&] { EGT_LAUNCH_CHECK(); return EGT_OK; }());
    // per-cloud cubes
    uint32_t* acc = nullptr;
    BTRY(cudaMallocAsync((void**)&acc, sizeof(uint32_t) * 6 * count, st));
    k_init_extents_batch<<<blocks(6 * count), kB, 0, st>>>(acc, count);
    k_extents_batch<<<blocks(N), kB, 0, st>>>(dxyz, N, b->d_cloud, acc);
    k_finalize_batch<<<blocks(count), kB, 0, st>>>(acc, cfg.eps, cfg.threshold, b->d_off, count, b->d_np);
    BSTAT([&] { for (int i = 0; i < 3; i++) count_launch(); EGT_CUDA_TRY(cudaGetLastError()); return EGT_OK; }());
    // normalise, key, one stable sort over (cloud, key), gather
    float4* tmp4 = nullptr;
    unsigned long long *kA = nullptr, *kB2 = nullptr;
    int *iA = nullptr, *iB = nullptr, *flag = nullptr, *cid = nullptr;
    BTRY(cudaMallocAsync((void**)&tmp4, sizeof(float4) * N, st));
    BTRY(cudaMallocAsync((void**)&kA, sizeof(unsigned long long) * N, st));
    BTRY(cudaMallocAsync((void**)&kB2, sizeof(unsigned long long) * N, st));
    BTRY(cudaMallocAsync((void**)&iA, sizeof(int) * N, st));
    BTRY(cudaMallocAsync((void**)&iB, sizeof(int) * N, st));
    BTRY(cudaMallocAsync((void**)&flag, sizeof(int) * N, st));
    BTRY(cudaMallocAsync((void**)&cid, sizeof(int) * N, st));
    const int end_bit = 30 + bits;
    size_t t_sort = 0, t_scan = 0;
    BTRY(cub::DeviceRadixSort::SortPairs(nullptr, t_sort, kA, kB2, iA, iB, N, 0, end_bit, st));
    BTRY(cub::DeviceScan::ExclusiveSum(nullptr, t_scan, flag, cid, (int)N, st));
    void* tmp = nullptr;
    BSTAT(scratch_reserve(h, std::max(t_sort, t_scan), &tmp));
    k_normalize_batch<<<blocks(N), kB, 0, st>>>(dxyz, N, b->d_cloud, b->d_np, tmp4, kA, iA);
    BSTAT([&] { EGT_LAUNCH_CHECK(); return EGT_OK; }());
    BTRY(cub::DeviceRadixSort::SortPairs(tmp, t_sort, kA, kB2, iA, iB, N, 0, end_bit, st));
    k_gather_batch<<<blocks(N), kB, 0, st>>>(tmp4, iB, N, b->d_cloud, b->d_off, b->d_np, h->p4, h->x, h->y, h->z,
                                            h->cell0, h->perm);
    BSTAT([&] { EGT_LAUNCH_CHECK(); return EGT_OK; }());
    BTRY(dev_alloc(h, &b->p4_input, sizeof(float4) * N));
    BTRY(cudaMemcpyAsync(b->p4_input, h->p4, sizeof(float4) * N, cudaMemcpyDeviceToDevice, st));
    // levels
    for (int L = 0; L < kMaxLevels; L++) {
        const int B = 1024 >> L;
        BTRY(dev_alloc(h, &b->cell_start[L], sizeof(int) * (N + count + 1)));
        BTRY(dev_alloc(h, &b->cell_x[L], sizeof(int) * (N + count + 1)));
        BTRY(dev_alloc(h, &b->rows[L], sizeof(int2) * (size_t)count * B * B));
        BTRY(dev_alloc(h, &b->cbase[L], sizeof(int) * count));
        BTRY(cudaMemsetAsync(b->rows[L], 0, sizeof(int2) * (size_t)count * B * B, st));
        const unsigned long long* keys = kB2;  // level 0: the sorted keys
        if (L > 0) {
            BTRY(dev_alloc(h, &b->order[L], sizeof(int) * N));
            k_level_key_batch<<<blocks(N), kB, 0, st>>>(h->cell0, b->d_cloud, b->d_off, N, L, kA, iA);
            BSTAT([&] { EGT_LAUNCH_CHECK(); return EGT_OK; }());
            BTRY(cub::DeviceRadixSort::SortPairs(tmp, t_sort, kA, kB2, iA, b->order[L], N, 0, end_bit, st));
            keys = kB2;
        }
        k_head_flags64<<<blocks(N), kB, 0, st>>>(keys, N, flag);
        BSTAT([&] { EGT_LAUNCH_CHECK(); return EGT_OK; }());
        BTRY(cub::DeviceScan::ExclusiveSum(tmp, t_scan, flag, cid, (int)N, st));
        k_cells_batch<<<blocks(N), kB, 0, st>>>(keys, flag, cid, b->d_cloud, b->d_off, N, B, L, b->cell_start[L],
                                               b->cell_x[L], b->rows[L], b->cbase[L], b->d_ctr);
        BSTAT([&] { EGT_LAUNCH_CHECK(); return EGT_OK; }());
    }
    DescArgs da{};
    da.p4 = h->p4;
    da.np = b->d_np;
    for (int L = 0; L < kMaxLevels; L++) {
        da.order[L] = b->order[L];
        da.cell_start[L] = b->cell_start[L];
        da.cell_x[L] = b->cell_x[L];
        da.rows[L] = b->rows[L];
        da.cbase[L] = b->cbase[L];
    }
    da.off = b->d_off;
    da.loff = b->d_loff;
    da.k = b->d_k;
    da.count = count;
    da.max_pts = cfg.max_points_in_cell;
    da.chunk = kChunk;
    da.lists = h->lists;
    da.kth = h->kth;
    da.qlevel = h->qlevel;
    da.ctr = b->d_ctr;
    k_make_desc<<<blocks(count), kB, 0, st>>>(da, b->d_desc);
    BSTAT([&] { EGT_LAUNCH_CHECK(); return EGT_OK; }());
    BTRY(cudaEventRecord(h->ev[1], st));
    for (void* p : {(void*)dxyz, (void*)acc, (void*)tmp4, (void*)kA, (void*)kB2, (void*)iA, (void*)iB, (void*)flag,
                    (void*)cid})
        cudaFreeAsync(p, st);
    BTRY(cudaStreamSynchronize(st));
    b->tm.grid_ms = elapsed_ms(h->ev[0], h->ev[1]);
    b->chunkoff_for = 0;
#undef BTRY
#undef BSTAT
    *out = b;
    return EGT_OK;
}

void egt_batch_destroy(egt_batch* b) {
    if (!b) return;
    cudaSetDevice(b->cfg.device);
    free_batch(b);
}

static egt_status batch_enter(egt_batch* b, void* stream) {
    if (!b) { set_error("null batch"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(b->cfg.device));
    b->h->stream = (cudaStream_t)stream;
    return EGT_OK;
}

egt_status egt_batch_knn(egt_batch* b, void* stream) {
    EGT_TRY(batch_enter(b, stream));
    return knn_batch(b);
}

egt_status egt_batch_filter(egt_batch* b, float alpha, void* stream) {
    EGT_TRY(batch_enter(b, stream));
    if (!(alpha > 0.f)) { set_error("egt_batch_filter: alpha must be > 0"); return EGT_ERR_ARG; }
    if (!b->have_knn) { set_error("egt_batch_filter: run egt_batch_knn first"); return EGT_ERR_STATE; }
    return filter_batch(b, alpha);
}

egt_status egt_batch_taubin(egt_batch* b, int iters, float lambda, float mu, void* stream) {
    EGT_TRY(batch_enter(b, stream));
    if (iters < 0) { set_error("egt_batch_taubin: iters must be >= 0"); return EGT_ERR_ARG; }
    if (!b->have_knn) { set_error("egt_batch_taubin: run egt_batch_knn first"); return EGT_ERR_STATE; }
    return taubin_batch(b, iters, lambda, mu);
}

egt_status egt_batch_set_tuning(egt_batch* b, int knn_chunk, int taubin_mode) {
    if (!b || knn_chunk < 1 || knn_chunk > 1024 || (taubin_mode != 0 && taubin_mode != 1)) {
        set_error("egt_batch_set_tuning: knn_chunk in [1, 1024], taubin_mode 0 or 1");
        return EGT_ERR_ARG;
    }
    b->chunk = knn_chunk;
    b->taubin_mode = taubin_mode;
    b->tuning_fixed = true;
    return EGT_OK;
}

egt_status egt_batch_run(egt_batch* b, int iters, float lambda, float mu, float alpha, void* stream) {
    EGT_TRY(batch_enter(b, stream));
    if (!(alpha > 0.f) || iters < 0) { set_error("egt_batch_run: alpha must be > 0 and iters >= 0"); return EGT_ERR_ARG; }
    // every run smooths the input clouds, whatever earlier calls did
    EGT_CUDA_TRY(cudaMemcpyAsync(b->h->p4, b->p4_input, sizeof(float4) * b->N, cudaMemcpyDeviceToDevice, b->h->stream));
    EGT_TRY(autotune(b, lambda, mu, alpha));
    if (b->kmax <= kFusedMaxK && b->fuse != 0) {
        EGT_TRY(knn_egt_batch(b, alpha));
    } else {
        b->tm.fused = 0;
        EGT_TRY(knn_batch(b));
        EGT_TRY(filter_batch(b, alpha));
    }
    return taubin_batch(b, iters, lambda, mu);
}

egt_status egt_batch_output(egt_batch* b, float* xyz_host, void* stream) {
    EGT_TRY(batch_enter(b, stream));
    if (!xyz_host) { set_error("egt_batch_output: null output"); return EGT_ERR_ARG; }
    egt_handle* h = b->h;
    cudaStream_t st = h->stream;
    float* d = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(float) * 3 * b->N, st));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[12], st));
    k_output_batch<<<blocks(b->N), kB, 0, st>>>(h->p4, h->perm, b->d_cloud, b->d_off, b->d_np, b->N, d);
    EGT_LAUNCH_CHECK();
    EGT_CUDA_TRY(cudaEventRecord(h->ev[13], st));
    EGT_CUDA_TRY(cudaMemcpyAsync(xyz_host, d, sizeof(float) * 3 * b->N, cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(d, st);
    EGT_CUDA_TRY(cudaStreamSynchronize(st));
    return EGT_OK;
}

egt_status egt_batch_get_knn_host(egt_batch* b, int cloud, int* lists_host) {
    if (!b || !lists_host || cloud < 0 || cloud >= b->count) { set_error("egt_batch_get_knn_host: bad argument"); return EGT_ERR_ARG; }
    if (!b->have_knn) { set_error("egt_batch_get_knn_host: run egt_batch_knn first"); return EGT_ERR_STATE; }
    EGT_CUDA_TRY(cudaSetDevice(b->cfg.device));
    egt_handle* h = b->h;
    cudaStream_t st = h->stream;
    const int n = (int)(b->off[cloud + 1] - b->off[cloud]);
    const int k = b->k[cloud];
    int* d = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(int) * (size_t)n * k, st));
    k_lists_cloud<<<blocks((int64_t)n * k), kB, 0, st>>>(h->lists + b->loff[cloud], h->perm + b->off[cloud], n, k, d);
    EGT_LAUNCH_CHECK();
    EGT_CUDA_TRY(cudaMemcpyAsync(lists_host, d, sizeof(int) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(d, st);
    EGT_CUDA_TRY(cudaStreamSynchronize(st));
    return EGT_OK;
}

egt_status egt_batch_get_timings(egt_batch* b, egt_batch_timings* t) {
    if (!b || !t) { set_error("egt_batch_get_timings: bad argument"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(b->cfg.device));
    egt_handle* h = b->h;
    EGT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    std::vector<unsigned long long> ctr((size_t)kCtrWords * b->count);
    EGT_CUDA_TRY(cudaMemcpy(ctr.data(), b->d_ctr, sizeof(unsigned long long) * ctr.size(), cudaMemcpyDeviceToHost));
    b->tm.knn_ms = elapsed_ms(h->ev[2], h->ev[3]);
    b->tm.egt_ms = elapsed_ms(h->ev[4], h->ev[5]);
    b->tm.taubin_ms = elapsed_ms(h->ev[6], h->ev[7]);
    b->tm.output_ms = elapsed_ms(h->ev[12], h->ev[13]);
    b->tm.clouds = b->count;
    b->tm.points = b->N;
    int64_t inv = 0, rer = 0;
    for (int c = 0; c < b->count; c++) {
        inv += (int64_t)ctr[(size_t)c * kCtrWords + kCtrInvalid];
        rer += (int64_t)ctr[(size_t)c * kCtrWords + kCtrExactRerun];
    }
    b->tm.invalid_queries = inv;
    b->tm.exact_reruns = rer;
    b->tm.csr_nnz = 0;
    if (b->have_csr) EGT_TRY(csr_nnz(h, &b->tm.csr_nnz));
    b->tm.knn_chunk = b->chunk > 0 ? b->chunk : kChunk;
    b->tm.taubin_mode = b->taubin_mode;
    *t = b->tm;
    return EGT_OK;
}

}  // extern "C"
