// Grid build: normalisation, level-0 cell sort and the cell hierarchy.
//
// Reference: GridStructure::InitStructure (GridKNNCuda.cu:1023-1133),
// getBuckets / InitializeLevel (GridKNNCuda.cu:898-946).
//
// Layout produced in HBM (all in cell-sorted order):
//   p4[n]      float4 (x,y,z,c) normalised positions; c = the packed level-0
//              cell coordinates (bit pattern), read together with the position
//   x/y/z[n]   SoA mirror                              -- KNNInterface views
//   cell0[n]   packed level-0 cell coords x|y<<10|z<<20
//   perm[n]    sorted slot -> original index
//   per level L (B = 1024 >> L):
//     order[n]          sorted indices grouped by level-L cell, ascending in a
//                       cell (level 0: identity, not stored)
//     cell_start[C+1]   cell -> [start,end) into order
//     cell_x[C]         x coordinate of the cell
//     row_range[B*B]    (y,z) row -> [first,last) cell, so a cell lookup is one
//                       row load plus a short binary search over x.
// Level-L cell = level-0 cell >> L exactly, because u*B_L = (u*1024)/2^L has no
// rounding; the hierarchy therefore never re-reads positions.
#include <cub/cub.cuh>
#include "egt_internal.cuh"
#include "grid_common.cuh"

namespace egt {
namespace {

// Per-axis min/max over AoS xyz (the six thrust::reduce calls of
// GridKNNCuda.cu:1042-1065 fused into one pass).
__global__ void k_extents(const float* __restrict__ xyz, int64_t n, uint32_t* __restrict__ acc) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            float v = xyz[3 * i + d];
            lo[d] = fminf(lo[d], v);
            hi[d] = fmaxf(hi[d], v);
        }
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
            hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            atomicMin(&acc[d], f2ord(lo[d]));
            atomicMax(&acc[3 + d], f2ord(hi[d]));
        }
    }
}

__global__ void k_init_extents(uint32_t* acc) {
    if (threadIdx.x < 3) acc[threadIdx.x] = 0xffffffffu;
    else if (threadIdx.x < 6) acc[threadIdx.x] = 0u;
}

// Scalar cube of InitStructure (finalize_norm in grid_common.cuh).
__global__ void k_finalize_norm(const uint32_t* acc, float eps, float thres0, int64_t n, NormParams* out) {
    *out = finalize_norm(acc, eps, thres0, n);
}

// GRIDCUDAKNNSELF_COMPACT's threshold scaling (GridKNNCuda.cu:2324-2325):
// thres /= (maxExtent - minExtent); thres *= thres.
__global__ void k_set_thres(float thres0, NormParams* np) {
    float t = __fdiv_rn(thres0, __fsub_rn(np->mx, np->mn));
    np->thres = __fmul_rn(t, t);
}

// normalize_points (GridKNNCuda.cu:840-849) + get_buckets_no_binary at B=1024
// (GridKNNCuda.cu:74-88): normalised float4 in original order and the key.
__global__ void k_normalize_key(const float* __restrict__ xyz, int64_t n, const NormParams* __restrict__ np,
                                float4* __restrict__ tmp4, uint32_t* __restrict__ key, int* __restrict__ idx) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const NormParams p = *np;
    const float d = __fsub_rn(p.mx, p.mn);
    float x = __fdiv_rn(__fsub_rn(xyz[3 * i], p.mn), d);
    float y = __fdiv_rn(__fsub_rn(xyz[3 * i + 1], p.mn), d);
    float z = __fdiv_rn(__fsub_rn(xyz[3 * i + 2], p.mn), d);
    tmp4[i] = make_float4(x, y, z, 0.f);
    int xi = cell_coord(x, p.a, p.b, 1024), yi = cell_coord(y, p.a, p.b, 1024), zi = cell_coord(z, p.a, p.b, 1024);
    key[i] = (uint32_t)(xi + yi * 1024 + zi * 1024 * 1024);
    idx[i] = (int)i;
}

// thrust::gather into sorted order (GridKNNCuda.cu:1114-1125) + SoA mirror.
__global__ void k_gather_sorted(const float4* __restrict__ tmp4, const int* __restrict__ perm, int64_t n,
                                float4* __restrict__ p4, float* __restrict__ x, float* __restrict__ y,
                                float* __restrict__ z, uint32_t* __restrict__ cell0,
                                const NormParams* __restrict__ np) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const NormParams p = *np;
    float4 v = tmp4[perm[s]];
    x[s] = v.x; y[s] = v.y; z[s] = v.z;
    uint32_t xi = cell_coord(v.x, p.a, p.b, 1024), yi = cell_coord(v.y, p.a, p.b, 1024),
             zi = cell_coord(v.z, p.a, p.b, 1024);
    const uint32_t packed = xi | (yi << 10) | (zi << 20);
    cell0[s] = packed;
    v.w = __uint_as_float(packed);  // the kNN reads a candidate's cell with its position
    p4[s] = v;
}

__global__ void k_level_key(const uint32_t* __restrict__ cell0, int64_t n, int L, uint32_t* __restrict__ key,
                            int* __restrict__ idx) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    uint32_t c = cell0[s];
    uint32_t B = 1024u >> L;
    uint32_t xi = (c & 1023u) >> L, yi = ((c >> 10) & 1023u) >> L, zi = ((c >> 20) & 1023u) >> L;
    key[s] = xi + yi * B + zi * B * B;
    idx[s] = (int)s;
}

__global__ void k_head_flags(const uint32_t* __restrict__ key, int64_t n, int* __restrict__ flag) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    flag[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}

// unique_by_key + cell starts (GridKNNCuda.cu:915-925), plus the row index:
// the head of cell c closes the row of cell c-1 when the rows differ.
__global__ void k_cells(const uint32_t* __restrict__ key, const int* __restrict__ flag,
                        const int* __restrict__ cid, int64_t n, int B, int* __restrict__ cell_start,
                        int* __restrict__ cell_x, int2* __restrict__ row_range, int* __restrict__ ncells) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t UB = (uint32_t)B;
    if (i == n - 1) {
        int nc = cid[i] + flag[i];
        *ncells = nc;
        cell_start[nc] = (int)n;
        row_range[key[i] / UB].y = nc;
    }
    if (!flag[i]) return;
    int c = cid[i];
    uint32_t k = key[i];
    cell_start[c] = (int)i;
    cell_x[c] = (int)(k % UB);
    uint32_t row = k / UB;
    if (c == 0) {
        row_range[row].x = 0;
    } else {
        uint32_t prow = key[i - 1] / UB;
        if (prow != row) {
            row_range[prow].y = c;
            row_range[row].x = c;
        }
    }
}

}  // namespace

egt_status scratch_reserve(egt_handle* h, size_t bytes, void** out) {
    if (h->scratch.bytes < bytes) {
        if (h->scratch.ptr) {
            dev_free(h, h->scratch.ptr);  // stream-ordered: pending work keeps it until done
            h->scratch.ptr = nullptr;
            h->scratch.bytes = 0;
        }
        size_t want = bytes + bytes / 4 + 256;
        EGT_CUDA_TRY(dev_alloc(h, &h->scratch.ptr, want));
        h->scratch.bytes = want;
    }
    *out = h->scratch.ptr;
    return EGT_OK;
}

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Builds the level tables 0..levels-1 for h (positions already sorted).
static egt_status build_levels(egt_handle* h, const uint32_t* sorted_key0, int levels) {
    const int64_t n = h->n;
    cudaStream_t st = h->stream;
    const int T = 256;
    const unsigned G = (unsigned)((n + T - 1) / T);
    // scratch: key in/out, idx in, flags, cid, cub temp
    size_t cub_sort = 0, cub_scan = 0;
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, cub_sort, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                                 (int*)nullptr, (int*)nullptr, (int)n, 0, 30, st));
    EGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, cub_scan, (int*)nullptr, (int*)nullptr, (int)n, st));
    size_t off_keyA = 0;
    size_t off_keyB = off_keyA + align256(4 * n);
    size_t off_idx = off_keyB + align256(4 * n);
    size_t off_flag = off_idx + align256(4 * n);
    size_t off_cid = off_flag + align256(4 * n);
    size_t off_cub = off_cid + align256(4 * n);
    size_t total = off_cub + align256(std::max(cub_sort, cub_scan));
    void* base = nullptr;
    EGT_TRY(scratch_reserve(h, total, &base));
    char* b = (char*)base;
    uint32_t* keyA = (uint32_t*)(b + off_keyA);
    uint32_t* keyB = (uint32_t*)(b + off_keyB);
    int* idx = (int*)(b + off_idx);
    int* flag = (int*)(b + off_flag);
    int* cid = (int*)(b + off_cid);
    void* cubtmp = b + off_cub;

    for (int L = 0; L < levels; L++) {
        LevelDev& lv = h->lv[L];
        lv.B = 1024 >> L;
        const uint32_t* key = nullptr;
        if (L == 0) {
            key = sorted_key0;
            lv.order = nullptr;
        } else {
            if (!lv.order) EGT_CUDA_TRY(dev_alloc(h, &lv.order, sizeof(int) * n));
            k_level_key<<<G, T, 0, st>>>(h->cell0, n, L, keyA, idx);
            EGT_LAUNCH_CHECK();
            size_t tb = cub_sort;
            EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(cubtmp, tb, keyA, keyB, idx, lv.order, (int)n, 0,
                                                         3 * (10 - L), st));
            key = keyB;
        }
        if (!lv.cell_start) EGT_CUDA_TRY(dev_alloc(h, &lv.cell_start, sizeof(int) * (n + 1)));
        if (!lv.cell_x) EGT_CUDA_TRY(dev_alloc(h, &lv.cell_x, sizeof(int) * n));
        if (!lv.row_range) EGT_CUDA_TRY(dev_alloc(h, &lv.row_range, sizeof(int2) * (size_t)lv.B * lv.B));
        EGT_CUDA_TRY(cudaMemsetAsync(lv.row_range, 0, sizeof(int2) * (size_t)lv.B * lv.B, st));
        k_head_flags<<<G, T, 0, st>>>(key, n, flag);
        EGT_LAUNCH_CHECK();
        size_t tb = cub_scan;
        EGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(cubtmp, tb, flag, cid, (int)n, st));
        k_cells<<<G, T, 0, st>>>(key, flag, cid, n, lv.B, lv.cell_start, lv.cell_x, lv.row_range,
                                 (int*)&h->d_counters[L]);
        EGT_LAUNCH_CHECK();
    }
    h->levels_built = levels;
    return EGT_OK;
}

// Full grid build from device AoS xyz (n points).  levels = number of
// hierarchy levels to build (8 for point clouds, 1 for meshes).
egt_status build_grid(egt_handle* h, const float* xyz, int levels) {
    const int64_t n = h->n;
    cudaStream_t st = h->stream;
    h->maxpop_valid = false;
    const int T = 256;
    const unsigned G = (unsigned)((n + T - 1) / T);
    EGT_CUDA_TRY(cudaEventRecord(h->ev[0], st));
    // extents
    uint32_t* acc = (uint32_t*)(h->d_counters + kCtrExtents);  // 6 words
    k_init_extents<<<1, 32, 0, st>>>(acc);
    EGT_LAUNCH_CHECK();
    unsigned ge = (unsigned)std::min<int64_t>((n + T - 1) / T, 148 * 8);
    if (ge == 0) ge = 1;
    k_extents<<<ge, T, 0, st>>>(xyz, n, acc);
    EGT_LAUNCH_CHECK();
    k_finalize_norm<<<1, 1, 0, st>>>(acc, h->cfg.eps, h->cfg.threshold, n, h->d_norm);
    EGT_LAUNCH_CHECK();
    // normalise + key + stable sort
    size_t cub_sort = 0;
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, cub_sort, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                                 (int*)nullptr, (int*)nullptr, (int)n, 0, 30, st));
    size_t off_tmp4 = 0;
    size_t off_kin = off_tmp4 + align256(16 * n);
    size_t off_kout = off_kin + align256(4 * n);
    size_t off_idx = off_kout + align256(4 * n);
    size_t off_cub = off_idx + align256(4 * n);
    size_t total = off_cub + align256(cub_sort);
    // The sorted key must survive into build_levels, which reuses scratch;
    // keep it in the handle's lists buffer region?  Use a dedicated buffer.
    uint32_t* key_sorted = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&key_sorted, sizeof(uint32_t) * n, st));
    void* base = nullptr;
    EGT_TRY(scratch_reserve(h, total, &base));
    char* b = (char*)base;
    float4* tmp4 = (float4*)(b + off_tmp4);
    uint32_t* kin = (uint32_t*)(b + off_kin);
    int* idx = (int*)(b + off_idx);
    void* cubtmp = b + off_cub;
    k_normalize_key<<<G, T, 0, st>>>(xyz, n, h->d_norm, tmp4, kin, idx);
    EGT_LAUNCH_CHECK();
    size_t tb = cub_sort;
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(cubtmp, tb, kin, key_sorted, idx, h->perm, (int)n, 0, 30, st));
    k_gather_sorted<<<G, T, 0, st>>>(tmp4, h->perm, n, h->p4, h->x, h->y, h->z, h->cell0, h->d_norm);
    EGT_LAUNCH_CHECK();
    egt_status s = build_levels(h, key_sorted, levels);
    cudaFreeAsync(key_sorted, st);
    EGT_TRY(s);
    EGT_CUDA_TRY(cudaMemcpyAsync(&h->norm, h->d_norm, sizeof(NormParams), cudaMemcpyDeviceToHost, st));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[1], st));
    return EGT_OK;
}

egt_status set_threshold(egt_handle* h, float thres) {
    k_set_thres<<<1, 1, 0, h->stream>>>(thres, h->d_norm);
    EGT_LAUNCH_CHECK();
    h->cfg.threshold = thres;
    return EGT_OK;
}

}  // namespace egt
