// Mesh 1-ring neighbour lists.
//
// Reference: GridMeshCuda::GetNeighborsFromTriangles (GridMeshCuda1.cu:416-511)
// with the kernel getMeshNeihbors (GridMeshCuda1.cu:99-138).  Every corner of
// every triangle offers the triangle's other two corners to its vertex's
// distance-sorted list, with the same admission rule as the grid kNN (strict
// '<' at slot k, dedup, FindPosition slot for equal distances).  The reference
// repeats full passes over all triangles, letting one triangle per vertex win
// an atomicExch flag per pass, until every corner has been consumed, so the
// order in which a vertex sees its triangles is decided by the scheduler.
//
// Here the corners are sorted by vertex once (stable, so ascending triangle
// order inside a vertex) and one warp per vertex inserts its candidates with
// the warp list of the grid kNN.  The produced sets are the reference's; the
// order of exactly equal distances follows ascending triangle index.
// Triangles with an index >= n are skipped (the reference maps them through
// an out-of-range read of its reverse permutation, GridMeshCuda1.cu:224-232).
#include <cub/cub.cuh>
#include "egt_internal.cuh"
#include "knn_common.cuh"

namespace egt {
namespace {

constexpr int kWarps = 8;

// reverseTriangleIndexes (GridMeshCuda1.cu:224-232) + corner keys.
__global__ void k_corners(const uint32_t* __restrict__ tris_orig, int64_t t, const int* __restrict__ rev, int n,
                          uint32_t* __restrict__ tris_sorted, uint32_t* __restrict__ ckey,
                          int* __restrict__ cid) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= t) return;
    uint32_t v[3];
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        v[c] = tris_orig[3 * i + c];
        ok &= v[c] < (uint32_t)n;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const uint32_t s = ok ? (uint32_t)rev[v[c]] : 0xffffffffu;
        tris_sorted[3 * i + c] = s;
        ckey[3 * i + c] = ok ? s : 0xffffffffu;  // invalid corners sort last
        cid[3 * i + c] = (int)(3 * i + c);
    }
}

__global__ void k_rev(const int* __restrict__ perm, int n, int* __restrict__ rev) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) rev[perm[s]] = s;
}

// Number of valid corners per vertex (exclusive-scanned into vertex ranges of
// the vertex-sorted corner array).
__global__ void k_vertex_hist(const uint32_t* __restrict__ ckey, int64_t m, int n, int* __restrict__ cnt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t v = ckey[i];
    if (v < (uint32_t)n) atomicAdd(&cnt[v], 1);
}

template <int S>
__global__ void __launch_bounds__(kWarps * 32) k_mesh_lists(const float4* __restrict__ p4,
                                                            const uint32_t* __restrict__ tris,
                                                            const int* __restrict__ corner,
                                                            const int* __restrict__ vstart, int n, int k,
                                                            int* __restrict__ lists) {
    const int lane = threadIdx.x & 31;
    const int v = blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (v >= n) return;
    const float4 pv = p4[v];
    WarpList<S> L;
    L.init(k);
    const int c0 = vstart[v], c1 = vstart[v + 1];
    for (int base = c0; base < c1; base += 16) {
        // each lane pair handles one corner: lane 2j -> first other corner, 2j+1 -> second
        const int e = base + (lane >> 1);
        float d = 0.f;
        int u = -1;
        if (e < c1) {
            const int cc = corner[e];
            const int tri = cc / 3, c = cc % 3;
            const int other = (lane & 1) ? (c == 2 ? 1 : 2) : (c == 0 ? 1 : 0);
            u = (int)tris[3 * (size_t)tri + other];
            const float4 q = p4[u];
            d = fs_dist3(pv.x, pv.y, pv.z, q.x, q.y, q.z);
        }
        unsigned mask = __ballot_sync(0xffffffffu, u >= 0 && d < L.kth);
        while (mask) {
            const int src = __ffs(mask) - 1;
            mask &= mask - 1;
            L.insert(__shfl_sync(0xffffffffu, d, src), __shfl_sync(0xffffffffu, u, src), lane);
        }
    }
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        if (t < k) lists[(size_t)v * k + t] = L.idx[s];
    }
}

template <int S>
egt_status launch_mesh(egt_handle* h, const int* corner, const int* vstart) {
    const unsigned G = (unsigned)((h->n + kWarps - 1) / kWarps);
    k_mesh_lists<S><<<G, kWarps * 32, 0, h->stream>>>(h->p4, h->tris, corner, vstart, (int)h->n, h->k, h->lists);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

}  // namespace

egt_status run_mesh_1ring(egt_handle* h, int k) {
    if (!h->is_mesh || !h->tris) { set_error("egt_mesh_1ring: handle has no triangles"); return EGT_ERR_STATE; }
    if (k <= 0 || k > 256) { set_error("egt_mesh_1ring: k must be in [1, 256]"); return EGT_ERR_ARG; }
    cudaStream_t st = h->stream;
    const int64_t n = h->n, t = h->t, m = 3 * t;
    if (h->k != k || !h->lists) {
        if (h->lists) dev_free(h, h->lists);
        h->lists = nullptr;
        EGT_CUDA_TRY(dev_alloc(h, &h->lists, sizeof(int) * (size_t)n * k));
        h->k = k;
    }
    h->have_csr = false;
    EGT_CUDA_TRY(cudaEventRecord(h->ev[2], st));
    // h->tris holds the ORIGINAL triangle indices until the first call; remap
    // them into sorted space and sort the corners by vertex.
    int* rev = nullptr;
    uint32_t *ckey = nullptr, *skey = nullptr, *tris_sorted = nullptr;
    int *cid = nullptr, *corner = nullptr, *vstart = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&rev, sizeof(int) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&ckey, sizeof(uint32_t) * std::max<int64_t>(m, 1), st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&skey, sizeof(uint32_t) * std::max<int64_t>(m, 1), st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&tris_sorted, sizeof(uint32_t) * std::max<int64_t>(m, 1), st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&cid, sizeof(int) * std::max<int64_t>(m, n + 1), st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&corner, sizeof(int) * std::max<int64_t>(m, 1), st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&vstart, sizeof(int) * (n + 1), st));
    k_rev<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(h->perm, (int)n, rev);
    EGT_LAUNCH_CHECK();
    if (m > 0) {
        k_corners<<<(unsigned)((t + 255) / 256), 256, 0, st>>>(h->tris, t, rev, (int)n, tris_sorted, ckey, cid);
        EGT_LAUNCH_CHECK();
        size_t tb = 0, ts = 0;
        EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, ckey, skey, cid, corner, (int)m, 0, 32, st));
        EGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, ts, (int*)nullptr, (int*)nullptr, (int)(n + 1), st));
        void* tmp = nullptr;
        EGT_TRY(scratch_reserve(h, std::max(tb, ts), &tmp));
        EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, ckey, skey, cid, corner, (int)m, 0, 32, st));
        // vertex ranges: histogram of valid corners, exclusive scan (cid is free again)
        EGT_CUDA_TRY(cudaMemsetAsync(cid, 0, sizeof(int) * (n + 1), st));
        k_vertex_hist<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(ckey, m, (int)n, cid);
        EGT_LAUNCH_CHECK();
        EGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, ts, cid, vstart, (int)(n + 1), st));
    } else {
        EGT_CUDA_TRY(cudaMemsetAsync(vstart, 0, sizeof(int) * (n + 1), st));
    }
    const uint32_t* tris_keep = h->tris;
    h->tris = tris_sorted;
    egt_status s;
    if (k <= 32) s = launch_mesh<1>(h, corner, vstart);
    else if (k <= 64) s = launch_mesh<2>(h, corner, vstart);
    else if (k <= 128) s = launch_mesh<4>(h, corner, vstart);
    else s = launch_mesh<8>(h, corner, vstart);
    h->tris = const_cast<uint32_t*>(tris_keep);
    EGT_CUDA_TRY(cudaEventRecord(h->ev[3], st));
    cudaFreeAsync(rev, st);
    cudaFreeAsync(ckey, st);
    cudaFreeAsync(skey, st);
    cudaFreeAsync(tris_sorted, st);
    cudaFreeAsync(cid, st);
    cudaFreeAsync(corner, st);
    cudaFreeAsync(vstart, st);
    return s;
}

}  // namespace egt
