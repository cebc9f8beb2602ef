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
// identical to the reference's), positions are float4 (one 16-byte gather per
// neighbour), the two ping-pong buffers stay in HBM/L2, and the 2*iters
// launches are captured once into a CUDA graph and replayed as one unit.
#include <algorithm>
#include "egt_internal.cuh"

namespace egt {
namespace {

// One half-step.  Each thread batches the column loads and position gathers of
// up to 8 neighbours (independent loads in flight), then accumulates them in
// list order.  The per-neighbour arithmetic is written exactly as the
// reference's expression and compiled with the same default contraction, so
// the rounding (and the result) is the reference's.
constexpr int kBatch = 8;

__global__ void __launch_bounds__(256) k_taubin(const float4* __restrict__ pin, float4* __restrict__ pout,
                                                const int* __restrict__ off, const int* __restrict__ col, int n,
                                                float scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = __ldg(pin + i);
    const float x1 = p.x, y1 = p.y, z1 = p.z;
    const int e0 = __ldg(off + i), e1 = __ldg(off + i + 1);
    float cog_x = 0.0f, cog_y = 0.0f, cog_z = 0.0f, sum = 0.0f;
    for (int e = e0; e < e1; e += kBatch) {
        const int cnt = min(kBatch, e1 - e);
        int j[kBatch];
        float4 q[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; u++) j[u] = u < cnt ? __ldg(col + e + u) : i;
#pragma unroll
        for (int u = 0; u < kBatch; u++) q[u] = __ldg(pin + j[u]);
#pragma unroll
        for (int u = 0; u < kBatch; u++) {
            if (u < cnt) {
                const float x2 = q[u].x, y2 = q[u].y, z2 = q[u].z;
                const float distance = (x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2) + (z1 - z2) * (z1 - z2);
                const float w = expf(-distance);
                cog_x += w * (x2 - x1);
                cog_y += w * (y2 - y1);
                cog_z += w * (z2 - z1);
                sum += w;
            }
        }
    }
    if (sum == 0.0f) sum = 1e-8f;
    float4 o;
    o.x = x1 + scale * cog_x / sum;
    o.y = y1 + scale * cog_y / sum;
    o.z = z1 + scale * cog_z / sum;
    o.w = 0.f;
    pout[i] = o;
}

__global__ void k_split_soa(const float4* __restrict__ p4, int n, float* __restrict__ x, float* __restrict__ y,
                            float* __restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = p4[i];
    x[i] = v.x; y[i] = v.y; z[i] = v.z;
}

}  // namespace

egt_status taubin_launch(const float4* pin, float4* pout, const int* off, const int* col, int n, float scale,
                         cudaStream_t st) {
    k_taubin<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(pin, pout, off, col, n, scale);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

egt_status run_taubin(egt_handle* h, int iters, float lambda, float mu) {
    if (iters < 0) { set_error("egt_taubin: iters must be >= 0"); return EGT_ERR_ARG; }
    if (!h->lists) { set_error("egt_taubin: no neighbour lists"); return EGT_ERR_STATE; }
    EGT_TRY(ensure_csr(h));
    cudaStream_t st = h->stream;
    const int n = (int)h->n;
    if (!h->p4b) EGT_CUDA_TRY(cudaMalloc(&h->p4b, sizeof(float4) * n));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[6], st));
    if (iters > 0) {
        const void* key[4] = {h->p4, h->p4b, h->csr_off, h->csr_col};
        const bool reuse = h->taubin_exec && h->taubin_iters == iters && h->taubin_lambda == lambda &&
                           h->taubin_mu == mu && std::equal(key, key + 4, h->taubin_key);
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
                    s = taubin_launch(h->p4, h->p4b, h->csr_off, h->csr_col, n, lambda, cap);
                    if (s == EGT_OK) s = taubin_launch(h->p4b, h->p4, h->csr_off, h->csr_col, n, mu, cap);
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
            h->taubin_lambda = lambda;
            h->taubin_mu = mu;
            std::copy(key, key + 4, h->taubin_key);
        } else {
            // the graph's launches are counted at capture; count the replayed ones too
            for (int i = 0; i < 2 * iters; i++) count_launch();
        }
        EGT_CUDA_TRY(cudaGraphLaunch(h->taubin_exec, st));
    }
    k_split_soa<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(h->p4, n, h->x, h->y, h->z);
    EGT_LAUNCH_CHECK();
    EGT_CUDA_TRY(cudaEventRecord(h->ev[7], st));
    return EGT_OK;
}

}  // namespace egt
