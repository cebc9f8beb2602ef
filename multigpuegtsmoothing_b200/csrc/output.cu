// Output gather and original-order exports.
//
// Reference: getOutputPoints (getOutputPoints.cu:9-63): x = x_hat*(max-min)+min,
// scattered from sorted slot s to original index perm[s]; and
// GridStructure::GetKNNIndexes (GridKNNCuda.cu:1941-1968, rearrangeReferenceNeighbors
// GridKNNCuda.cu:862-872): lists mapped to original ids and original row order.
#include "egt_internal.cuh"

namespace egt {
namespace {

__global__ void k_output(const float4* __restrict__ p4, const int* __restrict__ perm, int n,
                         const NormParams* __restrict__ np, float* __restrict__ x, float* __restrict__ y,
                         float* __restrict__ z) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float mn = np->mn, d = __fsub_rn(np->mx, np->mn);
    const float4 v = p4[s];
    const int o = perm[s];
    x[o] = __fmaf_rn(v.x, d, mn);
    y[o] = __fmaf_rn(v.y, d, mn);
    z[o] = __fmaf_rn(v.z, d, mn);
}

__global__ void k_lists_original(const int* __restrict__ lists, const int* __restrict__ perm, int n, int k,
                                 int* __restrict__ out) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * k) return;
    const int s = (int)(e / k), j = (int)(e % k);
    const int v = lists[e];
    out[(size_t)perm[s] * k + j] = v >= 0 ? perm[v] : -1;
}

__global__ void k_scatter3(const float* __restrict__ src, const int* __restrict__ perm, int n,
                           float* __restrict__ dst) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int o = perm[s];
    dst[o] = src[s];
    dst[n + o] = src[n + s];
    dst[2 * (size_t)n + o] = src[2 * (size_t)n + s];
}

}  // namespace

// rearrange_output (Normal_CUDA.cu:232-242 / getOutputPoints.cu:21-30): SoA
// sorted-space -> SoA original order.
egt_status scatter_original(egt_handle* h, const float* soa_sorted, float* soa_orig) {
    const int n = (int)h->n;
    k_scatter3<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(soa_sorted, h->perm, n, soa_orig);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

egt_status run_output(egt_handle* h, float* x, float* y, float* z) {
    const int n = (int)h->n;
    EGT_CUDA_TRY(cudaEventRecord(h->ev[12], h->stream));
    k_output<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(h->p4, h->perm, n, h->d_norm, x, y, z);
    EGT_LAUNCH_CHECK();
    EGT_CUDA_TRY(cudaEventRecord(h->ev[13], h->stream));
    return EGT_OK;
}

egt_status lists_original(egt_handle* h, int* out_dev) {
    const int64_t tot = h->n * (int64_t)h->k;
    k_lists_original<<<(unsigned)((tot + 255) / 256), 256, 0, h->stream>>>(h->lists, h->perm, (int)h->n, h->k,
                                                                          out_dev);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

}  // namespace egt
