// Taubin lambda/mu smoothing over the EGT-filtered CSR neighbourhoods.
//
// Reference: taubin_step_GKNN (EGT_CUDA.cu:229-276) driven by PerformSmoothing
// (EGT_CUDA.cu:559-633): per half-step
//     p' = p + s * sum_j w_j (q_j - p) / sum_j w_j,   w_j = expf(-|p - q_j|^2),
// s = lambda then mu, sum = 1e-8 when no neighbour contributes (isRegularized = 0,
// EGT_CUDA.cu:544).  The reference reads the full n*k list (including the -1
// entries the filter left) with three scalar gathers per neighbour, launches in
// 2M-thread chunks and synchronises after each of the 2*iters launches.
//
// Here: one thread per point walks its CSR row (kept neighbours only, in list
// order, so the floating-point accumulation order and therefore the result are
// identical to the reference's); positions are float4 (one 16-byte gather per
// neighbour); the 2*iters launches are captured once into a CUDA graph cached
// on the handle.  For the loop the working set is relabelled into Morton order
// of the level-0 cells: consecutive points then form compact 3-D blobs, so the
// neighbours of a 256-row tile are few and mostly inside the tile; each
// distinct neighbour position is gathered into shared memory once per tile and
// the rows read them from there.  Relabelling changes neither a row's neighbour order nor any value, so
// the result is the same bit for bit.
#include <algorithm>
#include <climits>
#include <cub/cub.cuh>
#include "egt_internal.cuh"

namespace egt {
namespace {

constexpr int kBatch = 8;        // neighbour gathers in flight per thread
constexpr int kTile = 256;       // rows per block
constexpr int kTileCap = 4608;   // CSR entries per staged tile (the 4M workload peaks at ~4.5k)

// One neighbour's contribution.  The squared distance is contracted as the
// reference build contracts norm2_GKNN inside taubin_step_GKNN --
// fma(dz,dz, fma(dy,dy, dx*dx)), found by comparing candidate contractions
// against the reference's own smoothed positions (0 mismatches on three
// fixtures).
__device__ __forceinline__ void accumulate(float x1, float y1, float z1, float4 q, float& cx, float& cy,
                                           float& cz, float& sum) {
    const float dx = __fsub_rn(x1, q.x), dy = __fsub_rn(y1, q.y), dz = __fsub_rn(z1, q.z);
    const float distance = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
    const float w = expf(-distance);
    cx = __fmaf_rn(w, __fsub_rn(q.x, x1), cx);
    cy = __fmaf_rn(w, __fsub_rn(q.y, y1), cy);
    cz = __fmaf_rn(w, __fsub_rn(q.z, z1), cz);
    sum = __fadd_rn(sum, w);
}

__device__ __forceinline__ float4 finish(float4 p, float cx, float cy, float cz, float sum, float scale) {
    if (sum == 0.0f) sum = 1e-8f;
    float4 o;
    o.x = __fadd_rn(p.x, __fdiv_rn(__fmul_rn(scale, cx), sum));
    o.y = __fadd_rn(p.y, __fdiv_rn(__fmul_rn(scale, cy), sum));
    o.z = __fadd_rn(p.z, __fdiv_rn(__fmul_rn(scale, cz), sum));
    o.w = p.w;  // keeps whatever the caller stores there (the packed cell coordinates)
    return o;
}

// Row walk with kBatch independent gathers in flight, accumulation in order.
// Entry e of the row is cols[e - cbase].
__device__ __forceinline__ float4 row_update(const float4* __restrict__ pin, const int* cols, int cbase, int e0,
                                             int e1, int self, float scale) {
    const float4 p = __ldg(pin + self);
    float cx = 0.0f, cy = 0.0f, cz = 0.0f, sum = 0.0f;
    for (int e = e0; e < e1; e += kBatch) {
        const int cnt = min(kBatch, e1 - e);
        int j[kBatch];
        float4 q[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; u++) j[u] = u < cnt ? cols[e + u - cbase] : self;
#pragma unroll
        for (int u = 0; u < kBatch; u++) q[u] = __ldg(pin + j[u]);
#pragma unroll
        for (int u = 0; u < kBatch; u++)
            if (u < cnt) accumulate(p.x, p.y, p.z, q[u], cx, cy, cz, sum);
    }
    return finish(p, cx, cy, cz, sum, scale);
}

// General half-step: any CSR, any point order (used by egt_taubin_noalloc).
__global__ void __launch_bounds__(256) k_taubin(const float4* __restrict__ pin, float4* __restrict__ pout,
                                                const int* __restrict__ off, const int* __restrict__ col, int n,
                                                float scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pout[i] = row_update(pin, col, 0, __ldg(off + i), __ldg(off + i + 1), i, scale);
}

// Staged half-step.  For every kTile-row tile the distinct neighbour indices
// (t_uni, precomputed once per CSR) are gathered into shared memory in one
// parallel pass, and every CSR entry carries its 16-bit index into that list
// (t_loc).  Rows then read their neighbours from shared memory in list order:
// each distinct position is fetched from global memory once per tile instead
// of once per reference.  Tiles whose lists would not fit (t_nu < 0) gather
// from global memory directly.
constexpr int kUCap = 1024;      // distinct neighbours staged per tile (16 KB; 99.8% of tiles fit)
constexpr size_t kStagedSmem = kUCap * sizeof(float4) + kTileCap * sizeof(uint16_t);

__global__ void __launch_bounds__(kTile, 6) k_taubin_staged(const float4* __restrict__ pin, float4* __restrict__ pout,
                                                         const int* __restrict__ off, const int* __restrict__ col,
                                                         const int* __restrict__ t_uni,
                                                         const uint16_t* __restrict__ t_loc,
                                                         const int* __restrict__ t_nu, int n, float scale) {
    extern __shared__ __align__(16) unsigned char smem[];
    float4* s_pos = reinterpret_cast<float4*>(smem);
    uint16_t* s_loc = reinterpret_cast<uint16_t*>(smem + kUCap * sizeof(float4));
    const int base = blockIdx.x * kTile;
    const int last = min(base + kTile, n);
    const int e_lo = __ldg(off + base), e_hi = __ldg(off + last);
    const int nu = __ldg(t_nu + blockIdx.x);
    if (nu >= 0) {
        for (int u = threadIdx.x; u < nu; u += kTile) s_pos[u] = __ldg(pin + __ldg(t_uni + e_lo + u));
        for (int t = threadIdx.x; t < e_hi - e_lo; t += kTile) s_loc[t] = __ldg(t_loc + e_lo + t);
    }
    __syncthreads();
    const int i = base + threadIdx.x;
    if (i >= n) return;
    if (nu < 0) {  // tile too large to stage: plain gathers
        const float4 p = __ldg(pin + i);
        float cx = 0.0f, cy = 0.0f, cz = 0.0f, sum = 0.0f;
        for (int e = __ldg(off + i); e < __ldg(off + i + 1); e++)
            accumulate(p.x, p.y, p.z, __ldg(pin + __ldg(col + e)), cx, cy, cz, sum);
        pout[i] = finish(p, cx, cy, cz, sum, scale);
        return;
    }
    const float4 p = __ldg(pin + i);
    const int e0 = __ldg(off + i) - e_lo, e1 = __ldg(off + i + 1) - e_lo;
    float cx = 0.0f, cy = 0.0f, cz = 0.0f, sum = 0.0f;
#pragma unroll 4
    for (int e = e0; e < e1; e++) accumulate(p.x, p.y, p.z, s_pos[s_loc[e]], cx, cy, cz, sum);
    pout[i] = finish(p, cx, cy, cz, sum, scale);
}

// Builds t_uni / t_loc / t_nu for one tile: block radix sort of the tile's
// column indices, unique, then each entry's position in the unique list.
constexpr int kBuildThreads = 512;
constexpr int kBuildItems = kTileCap / kBuildThreads;

__global__ void __launch_bounds__(kBuildThreads) k_tile_build(const int* __restrict__ off, const int* __restrict__ col,
                                                              int n, int* __restrict__ t_uni,
                                                              uint16_t* __restrict__ t_loc, int* __restrict__ t_nu) {
    using Sort = cub::BlockRadixSort<int, kBuildThreads, kBuildItems>;
    using Scan = cub::BlockScan<int, kBuildThreads>;
    __shared__ union {
        typename Sort::TempStorage sort;
        int uniq[kTileCap];
    } sm;
    __shared__ typename Scan::TempStorage scan;
    __shared__ int s_last[kBuildThreads];
    __shared__ int s_nu;
    const int base = blockIdx.x * kTile;
    const int last = min(base + kTile, n);
    const int e_lo = off[base], e_hi = off[last];
    const int cnt = e_hi - e_lo;
    if (cnt > kTileCap) {
        if (threadIdx.x == 0) t_nu[blockIdx.x] = -1;
        return;
    }
    int keys[kBuildItems];
#pragma unroll
    for (int j = 0; j < kBuildItems; j++) {
        const int i = threadIdx.x * kBuildItems + j;
        keys[j] = i < cnt ? col[e_lo + i] : INT_MAX;
    }
    Sort(sm.sort).Sort(keys);
    s_last[threadIdx.x] = keys[kBuildItems - 1];
    __syncthreads();
    int prev = threadIdx.x > 0 ? s_last[threadIdx.x - 1] : -1;
    int first[kBuildItems];
    int mine = 0;
#pragma unroll
    for (int j = 0; j < kBuildItems; j++) {
        first[j] = keys[j] != INT_MAX && keys[j] != prev;
        mine += first[j];
        prev = keys[j];
    }
    int at = 0, total = 0;
    Scan(scan).ExclusiveSum(mine, at, total);
    __syncthreads();  // the sort storage is reused for the unique list
#pragma unroll
    for (int j = 0; j < kBuildItems; j++)
        if (first[j]) sm.uniq[at++] = keys[j];
    if (threadIdx.x == 0) s_nu = total;
    __syncthreads();
    const int nu = s_nu;
    if (nu > kUCap) {
        if (threadIdx.x == 0) t_nu[blockIdx.x] = -1;
        return;
    }
    for (int u = threadIdx.x; u < nu; u += kBuildThreads) t_uni[e_lo + u] = sm.uniq[u];
    for (int i = threadIdx.x; i < cnt; i += kBuildThreads) {
        const int v = col[e_lo + i];
        int lo = 0, hi = nu - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (sm.uniq[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        t_loc[e_lo + i] = (uint16_t)lo;
    }
    if (threadIdx.x == 0) t_nu[blockIdx.x] = nu;
}

__global__ void k_split_soa(const float4* __restrict__ p4, int n, float* __restrict__ x, float* __restrict__ y,
                            float* __restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = p4[i];
    x[i] = v.x; y[i] = v.y; z[i] = v.z;
}

// 30-bit Morton code of a packed level-0 cell (x | y<<10 | z<<20).
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__global__ void k_morton_keys(const uint32_t* __restrict__ cell0, int n, uint32_t* __restrict__ key,
                              int* __restrict__ idx) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t c = cell0[s];
    key[s] = spread3(c) | (spread3(c >> 10) << 1) | (spread3(c >> 20) << 2);
    idx[s] = s;
}

// Batched clouds: the cloud id above the Morton key keeps each cloud's rows together.
__global__ void k_morton_keys64(const uint32_t* __restrict__ cell0, const uint16_t* __restrict__ cloud, int n,
                                unsigned long long* __restrict__ key, int* __restrict__ idx) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t c = cell0[s];
    key[s] = ((unsigned long long)cloud[s] << 30) | (spread3(c) | (spread3(c >> 10) << 1) | (spread3(c >> 20) << 2));
    idx[s] = s;
}

__global__ void k_morton_rows(const int* __restrict__ perm, const int* __restrict__ off, int n, int* __restrict__ inv,
                              int* __restrict__ len) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) { len[n] = 0; return; }
    const int s = perm[i];
    inv[s] = i;
    len[i] = off[s + 1] - off[s];
}

__global__ void k_morton_cols(const int* __restrict__ perm, const int* __restrict__ inv, const int* __restrict__ off,
                              const int* __restrict__ col, const int* __restrict__ moff, int n,
                              int* __restrict__ mcol) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = perm[i];
    const int e0 = off[s], e1 = off[s + 1], o = moff[i];
    for (int e = e0; e < e1; e++) mcol[o + (e - e0)] = inv[col[e]];
}

__global__ void k_gather_morton(const float4* __restrict__ p4, const int* __restrict__ perm, int n,
                                float4* __restrict__ mp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) mp[i] = p4[perm[i]];
}

__global__ void k_scatter_morton(const float4* __restrict__ mp, const int* __restrict__ perm, int n,
                                 float4* __restrict__ p4, float* __restrict__ x, float* __restrict__ y,
                                 float* __restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = mp[i];
    const int s = perm[i];
    p4[s] = v;
    x[s] = v.x; y[s] = v.y; z[s] = v.z;
}

}  // namespace

egt_status taubin_launch(const float4* pin, float4* pout, const int* off, const int* col, int n, float scale,
                         cudaStream_t st) {
    k_taubin<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(pin, pout, off, col, n, scale);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

static egt_status staged_launch(egt_handle* h, const float4* pin, float4* pout, float scale, cudaStream_t st) {
    const int n = (int)h->n;
    k_taubin_staged<<<(unsigned)((n + kTile - 1) / kTile), kTile, kStagedSmem, st>>>(
        pin, pout, h->m_off, h->m_col, h->t_uni, h->t_loc, h->t_nu, n, scale);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

// Builds the Morton-order copy of the CSR (when the CSR changed) and gathers
// the current positions into Morton order.
static egt_status morton_prepare(egt_handle* h) {
    cudaStream_t st = h->stream;
    const int n = (int)h->n;
    const unsigned G = (unsigned)((n + 256) / 256);
    if (!h->m_perm) {
        EGT_CUDA_TRY(dev_alloc(h, &h->m_perm, sizeof(int) * n));
        EGT_CUDA_TRY(dev_alloc(h, &h->m_inv, sizeof(int) * n));
        EGT_CUDA_TRY(dev_alloc(h, &h->m_p, sizeof(float4) * n));
        EGT_CUDA_TRY(dev_alloc(h, &h->m_pb, sizeof(float4) * n));
        EGT_CUDA_TRY(dev_alloc(h, &h->m_off, sizeof(int) * (n + 1)));
    }
    if (h->m_version != h->csr_version) {
        int64_t nnz = 0;
        EGT_TRY(csr_nnz(h, &nnz));  // one host round trip per CSR, at set-up
        if (h->m_cap < nnz || !h->m_col) {
            if (h->m_col) dev_free(h, h->m_col);
            h->m_col = nullptr;
            EGT_CUDA_TRY(dev_alloc(h, &h->m_col, sizeof(int) * std::max<int64_t>(nnz, 1)));
            h->m_cap = std::max<int64_t>(nnz, 1);
        }
        // keys: 30-bit Morton code of the level-0 cell, below the cloud id for batches
        const bool wide = h->cloud_of != nullptr;
        const int end_bit = wide ? 30 + h->cloud_bits : 30;
        const size_t kb = wide ? sizeof(unsigned long long) : sizeof(uint32_t);
        void *kin = nullptr, *kout = nullptr;
        int *idx = nullptr, *len = nullptr;
        EGT_CUDA_TRY(cudaMallocAsync(&kin, kb * n, st));
        EGT_CUDA_TRY(cudaMallocAsync(&kout, kb * n, st));
        EGT_CUDA_TRY(cudaMallocAsync((void**)&idx, sizeof(int) * n, st));
        EGT_CUDA_TRY(cudaMallocAsync((void**)&len, sizeof(int) * (n + 1), st));
        if (wide) k_morton_keys64<<<G, 256, 0, st>>>(h->cell0, h->cloud_of, n, (unsigned long long*)kin, idx);
        else k_morton_keys<<<G, 256, 0, st>>>(h->cell0, n, (uint32_t*)kin, idx);
        EGT_LAUNCH_CHECK();
        size_t t_sort = 0, t_scan = 0;
        if (wide)
            EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, t_sort, (unsigned long long*)kin,
                                                         (unsigned long long*)kout, idx, h->m_perm, n, 0, end_bit, st));
        else
            EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, t_sort, (uint32_t*)kin, (uint32_t*)kout, idx,
                                                         h->m_perm, n, 0, end_bit, st));
        EGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, t_scan, len, h->m_off, n + 1, st));
        void* tmp = nullptr;
        EGT_TRY(scratch_reserve(h, std::max(t_sort, t_scan), &tmp));
        if (wide)
            EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, t_sort, (unsigned long long*)kin,
                                                         (unsigned long long*)kout, idx, h->m_perm, n, 0, end_bit, st));
        else
            EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, t_sort, (uint32_t*)kin, (uint32_t*)kout, idx,
                                                         h->m_perm, n, 0, end_bit, st));
        k_morton_rows<<<G, 256, 0, st>>>(h->m_perm, h->csr_off, n, h->m_inv, len);
        EGT_LAUNCH_CHECK();
        EGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, t_scan, len, h->m_off, n + 1, st));
        k_morton_cols<<<G, 256, 0, st>>>(h->m_perm, h->m_inv, h->csr_off, h->csr_col, h->m_off, n, h->m_col);
        EGT_LAUNCH_CHECK();
        // per-tile distinct-neighbour lists for the staged half-step
        const unsigned tiles = (unsigned)((n + kTile - 1) / kTile);
        if (h->t_uni) dev_free(h, h->t_uni);
        if (h->t_loc) dev_free(h, h->t_loc);
        if (h->t_nu) dev_free(h, h->t_nu);
        h->t_uni = nullptr; h->t_loc = nullptr; h->t_nu = nullptr;
        EGT_CUDA_TRY(dev_alloc(h, &h->t_uni, sizeof(int) * std::max<int64_t>(nnz, 1)));
        EGT_CUDA_TRY(dev_alloc(h, &h->t_loc, sizeof(uint16_t) * std::max<int64_t>(nnz, 1)));
        EGT_CUDA_TRY(dev_alloc(h, &h->t_nu, sizeof(int) * tiles));
        k_tile_build<<<tiles, kBuildThreads, 0, st>>>(h->m_off, h->m_col, n, h->t_uni, h->t_loc, h->t_nu);
        EGT_LAUNCH_CHECK();
        cudaFreeAsync(kin, st);
        cudaFreeAsync(kout, st);
        cudaFreeAsync(idx, st);
        cudaFreeAsync(len, st);
        h->m_version = h->csr_version;
    }
    k_gather_morton<<<G, 256, 0, st>>>(h->p4, h->m_perm, n, h->m_p);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

egt_status run_taubin(egt_handle* h, int iters, float lambda, float mu) {
    if (iters < 0) { set_error("egt_taubin: iters must be >= 0"); return EGT_ERR_ARG; }
    if (!h->lists) { set_error("egt_taubin: no neighbour lists"); return EGT_ERR_STATE; }
    EGT_TRY(ensure_csr(h));
    cudaStream_t st = h->stream;
    const int n = (int)h->n;
    EGT_CUDA_TRY(cudaEventRecord(h->ev[6], st));
    if (iters > 0) {
        EGT_TRY(morton_prepare(h));
        static bool smem_set = false;
        if (!smem_set) {
            EGT_CUDA_TRY(cudaFuncSetAttribute(k_taubin_staged, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)kStagedSmem));
            smem_set = true;
        }
        const void* key[4] = {h->m_p, h->m_pb, h->t_uni, h->t_loc};
        const bool reuse = h->taubin_exec && h->taubin_iters == iters && h->taubin_lambda == lambda &&
                           h->taubin_mu == mu && h->taubin_graph_mode == h->taubin_mode &&
                           std::equal(key, key + 4, h->taubin_key);
        if (!reuse) {
            if (h->taubin_exec) { cudaGraphExecDestroy(h->taubin_exec); h->taubin_exec = nullptr; }
            // capture the 2*iters half-steps once; replays reuse the executable graph
            cudaGraph_t g = nullptr;
            cudaStream_t cap = nullptr;
            EGT_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            egt_status s = EGT_OK;
            cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                for (int it = 0; it < iters && s == EGT_OK; it++) {
                    if (h->taubin_mode == 0) {
                        s = staged_launch(h, h->m_p, h->m_pb, lambda, cap);
                        if (s == EGT_OK) s = staged_launch(h, h->m_pb, h->m_p, mu, cap);
                    } else {  // direct gathers (no tile staging)
                        s = taubin_launch(h->m_p, h->m_pb, h->m_off, h->m_col, n, lambda, cap);
                        if (s == EGT_OK) s = taubin_launch(h->m_pb, h->m_p, h->m_off, h->m_col, n, mu, cap);
                    }
                }
                cudaError_t e2 = cudaStreamEndCapture(cap, &g);
                if (e2 != cudaSuccess && s == EGT_OK) { set_error(cuda_msg(e2, "EndCapture", __FILE__, __LINE__)); s = EGT_ERR_CUDA; }
            } else {
                set_error(cuda_msg(e, "BeginCapture", __FILE__, __LINE__));
                s = EGT_ERR_CUDA;
            }
            if (s == EGT_OK) {
                e = cudaGraphInstantiate(&h->taubin_exec, g, 0);
                if (e != cudaSuccess) {
                    set_error(cuda_msg(e, "GraphInstantiate", __FILE__, __LINE__));
                    h->taubin_exec = nullptr;
                    s = EGT_ERR_CUDA;
                }
            }
            if (g) cudaGraphDestroy(g);
            cudaStreamDestroy(cap);
            EGT_TRY(s);
            h->taubin_iters = iters;
            h->taubin_graph_mode = h->taubin_mode;
            h->taubin_lambda = lambda;
            h->taubin_mu = mu;
            std::copy(key, key + 4, h->taubin_key);
        } else {
            // the graph's launches are counted at capture; count the replayed ones too
            for (int i = 0; i < 2 * iters; i++) count_launch();
        }
        EGT_CUDA_TRY(cudaGraphLaunch(h->taubin_exec, st));
        k_scatter_morton<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(h->m_p, h->m_perm, n, h->p4, h->x, h->y,
                                                                       h->z);
        EGT_LAUNCH_CHECK();
    } else {
        k_split_soa<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(h->p4, n, h->x, h->y, h->z);
        EGT_LAUNCH_CHECK();
    }
    EGT_CUDA_TRY(cudaEventRecord(h->ev[7], st));
    return EGT_OK;
}

}  // namespace egt
