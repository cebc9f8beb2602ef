// Learned search proposal: features, labels, the proposal network's
// inference and training kernels, and the egt_proposal_* entry points.
//
// An extension of this project; the reference has no counterpart.  The
// network is an MLP 8 -> 32 -> 32 -> 16 with ReLU activations and a softmax
// over the 16 classes of proposal.cuh.  Its parameters are stored as binary16
// and every kernel computes with those values in FP32 (FP32 accumulation);
// training keeps FP32 master copies and Adam moments and re-rounds the
// binary16 parameters after each step.  The loss is the mean cross-entropy
// against labels derived from the plain grid kNN: the cheapest box that
// contains the query's k-th distance ball (with the certification margin).
#include <cuda_fp16.h>

#include <cmath>
#include <vector>

#include "proposal.cuh"

struct egt_proposal {
    int device = 0;
    int k = 0;
    uint64_t seed = 0;
    cudaStream_t stream = nullptr;
    __half* params = nullptr;  // [kPropParams] binary16 parameters
    float* master = nullptr;   // [kPropParams] FP32 master copy
    float* m1 = nullptr;       // Adam moments
    float* m2 = nullptr;
    float* grad = nullptr;     // [kPropParams] gradient accumulator
    float* loss = nullptr;     // [loss_cap] per-step loss
    int64_t loss_cap = 0;
    float* feats = nullptr;    // [cap * 8] training features
    uint8_t* labels = nullptr; // [cap]
    int64_t m = 0, cap = 0;
    int64_t step = 0;          // Adam steps taken
    float tau = 0.85f;
};

namespace egt {
namespace {

constexpr int kTB = 128;  // training samples per block

// ---------------------------------------------------------------------------
// Network forward pass for one sample.  w: parameters (binary16 values held
// as float in shared memory); weights are read four at a time.
__device__ __forceinline__ void mlp_forward(const float* __restrict__ w, const float x[kPropFeatures],
                                            float h1[kPropHidden], float h2[kPropHidden], float z[kPropClasses]) {
#pragma unroll
    for (int o = 0; o < kPropHidden; o++) {
        const float4* r = reinterpret_cast<const float4*>(w + kPW1 + o * kPropFeatures);
        float acc = w[kPB1 + o];
#pragma unroll
        for (int i = 0; i < kPropFeatures / 4; i++) {
            const float4 v = r[i];
            acc = fmaf(v.x, x[4 * i], acc);
            acc = fmaf(v.y, x[4 * i + 1], acc);
            acc = fmaf(v.z, x[4 * i + 2], acc);
            acc = fmaf(v.w, x[4 * i + 3], acc);
        }
        h1[o] = fmaxf(acc, 0.0f);
    }
#pragma unroll
    for (int o = 0; o < kPropHidden; o++) {
        const float4* r = reinterpret_cast<const float4*>(w + kPW2 + o * kPropHidden);
        float acc = w[kPB2 + o];
#pragma unroll
        for (int i = 0; i < kPropHidden / 4; i++) {
            const float4 v = r[i];
            acc = fmaf(v.x, h1[4 * i], acc);
            acc = fmaf(v.y, h1[4 * i + 1], acc);
            acc = fmaf(v.z, h1[4 * i + 2], acc);
            acc = fmaf(v.w, h1[4 * i + 3], acc);
        }
        h2[o] = fmaxf(acc, 0.0f);
    }
#pragma unroll
    for (int c = 0; c < kPropClasses; c++) {
        const float4* r = reinterpret_cast<const float4*>(w + kPW3 + c * kPropHidden);
        float acc = w[kPB3 + c];
#pragma unroll
        for (int i = 0; i < kPropHidden / 4; i++) {
            const float4 v = r[i];
            acc = fmaf(v.x, h2[4 * i], acc);
            acc = fmaf(v.y, h2[4 * i + 1], acc);
            acc = fmaf(v.z, h2[4 * i + 2], acc);
            acc = fmaf(v.w, h2[4 * i + 3], acc);
        }
        z[c] = acc;
    }
}

__device__ __forceinline__ void load_params(const __half* __restrict__ params, float* w) {
    for (int i = threadIdx.x; i < kPropParams; i += blockDim.x) w[i] = __half2float(params[i]);
}

struct ProposeArgs {
    const float4* __restrict__ p4;
    const NormParams* __restrict__ np;
    LevelDev lv[kMaxLevels];
    int n;
    int stride;                       // query q = j * stride for thread j
    const __half* __restrict__ params;
    float tau;
    float* __restrict__ feats;        // optional [rows * 8]
    uint8_t* __restrict__ cls;        // optional [n] proposed class per query
    const float* __restrict__ kth;    // optional: labels from the plain k-th distance
    uint8_t* __restrict__ labels;     // optional [rows]
};

// Features (+ label) (+ class) of queries j * stride, one thread each.
__global__ void __launch_bounds__(256) k_propose(ProposeArgs a) {
    __shared__ __align__(16) float w[kPropParams];
    if (a.cls) load_params(a.params, w);
    __syncthreads();
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t q = j * a.stride;
    if (q >= a.n) return;
    const NormParams np = *a.np;
    const float4 pq = a.p4[q];
    float f[kPropFeatures];
    proposal_features(a.lv, np, pq, f);
    if (a.feats) {
        float4* dst = reinterpret_cast<float4*>(a.feats + j * kPropFeatures);
        dst[0] = make_float4(f[0], f[1], f[2], f[3]);
        dst[1] = make_float4(f[4], f[5], f[6], f[7]);
    }
    if (a.labels) {
        const float kk = a.kth[q];
        int lab = kPropPlain;
        if (kk < 1e10f) {
            const uint32_t c0 = __float_as_uint(pq.w);
            for (int c = 0; c < kPropPlain; c++) {
                int lo[3], end[3];
                box_bounds(c, kBoxClass[c][1], c0, lo, end);
                if (ball_in_box(np, pq, kk, lo, end)) { lab = c; break; }
            }
        }
        a.labels[j] = (uint8_t)lab;
    }
    if (a.cls) {
        float h1[kPropHidden], h2[kPropHidden], z[kPropClasses];
        mlp_forward(w, f, h1, h2, z);
        float mx = z[0];
#pragma unroll
        for (int c = 1; c < kPropClasses; c++) mx = fmaxf(mx, z[c]);
        float sum = 0.0f;
#pragma unroll
        for (int c = 0; c < kPropClasses; c++) { z[c] = expf(z[c] - mx); sum += z[c]; }
        const float thr = a.tau * sum;
        float cum = 0.0f;
        int cls = kPropPlain;
#pragma unroll
        for (int c = 0; c < kPropClasses; c++) {
            cum += z[c];
            if (cum >= thr && cls == kPropPlain) cls = c;
        }
        a.cls[q] = (uint8_t)cls;
    }
}

// ---------------------------------------------------------------------------
// Training.  One block runs forward + backward for kTB samples (one per
// thread), keeps the activations and deltas in shared memory and reduces the
// parameter gradients over its samples before one atomicAdd per parameter.

__device__ __forceinline__ uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct TrainArgs {
    const __half* __restrict__ params;
    const float* __restrict__ feats;
    const uint8_t* __restrict__ labels;
    int64_t m;         // samples available
    int batch;         // samples in this step
    uint64_t seed;
    int64_t step;
    int sequential;    // 1: sample j is row j (gradient checks); 0: drawn with replacement
    float* __restrict__ grad;
    float* __restrict__ loss;  // this step's loss slot
};

constexpr int kSX = kPropFeatures + 1, kSH = kPropHidden + 1, kSZ = kPropClasses + 1;
constexpr size_t kTrainSmem =
    sizeof(float) * (kPropParams + kTB * (kSX + 4 * kSH + kSZ) + kTB / 32);

__global__ void __launch_bounds__(kTB) k_train_batch(TrainArgs t) {
    extern __shared__ __align__(16) float sm[];
    float* w = sm;
    float* sx = w + kPropParams;
    float* sh1 = sx + kTB * kSX;
    float* sh2 = sh1 + kTB * kSH;
    float* sd1 = sh2 + kTB * kSH;
    float* sd2 = sd1 + kTB * kSH;
    float* sd3 = sd2 + kTB * kSH;
    float* sloss = sd3 + kTB * kSZ;
    load_params(t.params, w);
    __syncthreads();
    const int tid = threadIdx.x;
    const int64_t j = (int64_t)blockIdx.x * kTB + tid;
    const bool valid = j < t.batch;
    const float inv_b = 1.0f / (float)t.batch;
    float* rx = sx + tid * kSX;
    float* rh1 = sh1 + tid * kSH;
    float* rh2 = sh2 + tid * kSH;
    float* rd1 = sd1 + tid * kSH;
    float* rd2 = sd2 + tid * kSH;
    float* rd3 = sd3 + tid * kSZ;
    int y = 0;
    {
        float x[kPropFeatures];
        if (valid) {
            const int64_t s = t.sequential ? j
                                           : (int64_t)(mix64(t.seed ^ mix64((uint64_t)t.step * 0x100000001B3ull + j)) %
                                                       (uint64_t)t.m);
            const float4* src = reinterpret_cast<const float4*>(t.feats + s * kPropFeatures);
            const float4 a0 = src[0], a1 = src[1];
            x[0] = a0.x; x[1] = a0.y; x[2] = a0.z; x[3] = a0.w;
            x[4] = a1.x; x[5] = a1.y; x[6] = a1.z; x[7] = a1.w;
            y = t.labels[s];
        } else {
#pragma unroll
            for (int i = 0; i < kPropFeatures; i++) x[i] = 0.0f;
        }
#pragma unroll
        for (int i = 0; i < kPropFeatures; i++) rx[i] = x[i];
        // layer 1
#pragma unroll 4
        for (int o = 0; o < kPropHidden; o++) {
            float acc = w[kPB1 + o];
#pragma unroll
            for (int i = 0; i < kPropFeatures; i++) acc = fmaf(w[kPW1 + o * kPropFeatures + i], x[i], acc);
            rh1[o] = fmaxf(acc, 0.0f);
        }
    }
    // layer 2
    {
        float h1[kPropHidden];
#pragma unroll
        for (int i = 0; i < kPropHidden; i++) h1[i] = rh1[i];
#pragma unroll 2
        for (int o = 0; o < kPropHidden; o++) {
            const float4* r = reinterpret_cast<const float4*>(w + kPW2 + o * kPropHidden);
            float acc = w[kPB2 + o];
#pragma unroll
            for (int i = 0; i < kPropHidden / 4; i++) {
                const float4 v = r[i];
                acc = fmaf(v.x, h1[4 * i], acc);
                acc = fmaf(v.y, h1[4 * i + 1], acc);
                acc = fmaf(v.z, h1[4 * i + 2], acc);
                acc = fmaf(v.w, h1[4 * i + 3], acc);
            }
            rh2[o] = fmaxf(acc, 0.0f);
        }
    }
    // layer 3, softmax, loss and d loss / d logits = (softmax - onehot) / batch
    float li = 0.0f;
    {
        float h2[kPropHidden], z[kPropClasses];
#pragma unroll
        for (int i = 0; i < kPropHidden; i++) h2[i] = rh2[i];
#pragma unroll
        for (int c = 0; c < kPropClasses; c++) {
            const float4* r = reinterpret_cast<const float4*>(w + kPW3 + c * kPropHidden);
            float acc = w[kPB3 + c];
#pragma unroll
            for (int i = 0; i < kPropHidden / 4; i++) {
                const float4 v = r[i];
                acc = fmaf(v.x, h2[4 * i], acc);
                acc = fmaf(v.y, h2[4 * i + 1], acc);
                acc = fmaf(v.z, h2[4 * i + 2], acc);
                acc = fmaf(v.w, h2[4 * i + 3], acc);
            }
            z[c] = acc;
        }
        float mx = z[0];
#pragma unroll
        for (int c = 1; c < kPropClasses; c++) mx = fmaxf(mx, z[c]);
        float sum = 0.0f, zy = 0.0f;
#pragma unroll
        for (int c = 0; c < kPropClasses; c++) {
            if (c == y) zy = z[c];
            z[c] = expf(z[c] - mx);
            sum += z[c];
        }
        li = valid ? logf(sum) - (zy - mx) : 0.0f;
#pragma unroll
        for (int c = 0; c < kPropClasses; c++)
            rd3[c] = valid ? (z[c] / sum - (c == y ? 1.0f : 0.0f)) * inv_b : 0.0f;
    }
    // back through layer 3
    {
        float d3[kPropClasses];
#pragma unroll
        for (int c = 0; c < kPropClasses; c++) d3[c] = rd3[c];
#pragma unroll 4
        for (int o = 0; o < kPropHidden; o++) {
            float acc = 0.0f;
#pragma unroll
            for (int c = 0; c < kPropClasses; c++) acc = fmaf(w[kPW3 + c * kPropHidden + o], d3[c], acc);
            rd2[o] = rh2[o] > 0.0f ? acc : 0.0f;
        }
    }
    // back through layer 2
    {
        float d2[kPropHidden];
#pragma unroll
        for (int i = 0; i < kPropHidden; i++) d2[i] = rd2[i];
#pragma unroll 2
        for (int o = 0; o < kPropHidden; o++) {
            float acc = 0.0f;
#pragma unroll
            for (int i = 0; i < kPropHidden; i++) acc = fmaf(w[kPW2 + i * kPropHidden + o], d2[i], acc);
            rd1[o] = rh1[o] > 0.0f ? acc : 0.0f;
        }
    }
    float lw = li;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lw += __shfl_xor_sync(0xffffffffu, lw, o);
    if ((tid & 31) == 0) sloss[tid >> 5] = lw;
    __syncthreads();
    const int rows = (int)min((int64_t)kTB, (int64_t)t.batch - (int64_t)blockIdx.x * kTB);
    for (int p = tid; p < kPropParams; p += kTB) {
        float g = 0.0f;
        if (p < kPB1) {
            const int o = p / kPropFeatures, i = p % kPropFeatures;
            for (int s = 0; s < rows; s++) g = fmaf(sd1[s * kSH + o], sx[s * kSX + i], g);
        } else if (p < kPW2) {
            const int o = p - kPB1;
            for (int s = 0; s < rows; s++) g += sd1[s * kSH + o];
        } else if (p < kPB2) {
            const int o = (p - kPW2) / kPropHidden, i = (p - kPW2) % kPropHidden;
            for (int s = 0; s < rows; s++) g = fmaf(sd2[s * kSH + o], sh1[s * kSH + i], g);
        } else if (p < kPW3) {
            const int o = p - kPB2;
            for (int s = 0; s < rows; s++) g += sd2[s * kSH + o];
        } else if (p < kPB3) {
            const int c = (p - kPW3) / kPropHidden, i = (p - kPW3) % kPropHidden;
            for (int s = 0; s < rows; s++) g = fmaf(sd3[s * kSZ + c], sh2[s * kSH + i], g);
        } else {
            const int c = p - kPB3;
            for (int s = 0; s < rows; s++) g += sd3[s * kSZ + c];
        }
        atomicAdd(&t.grad[p], g);
    }
    if (tid == 0) {
        float bl = 0.0f;
        for (int i = 0; i < kTB / 32; i++) bl += sloss[i];
        atomicAdd(t.loss, bl * inv_b);
    }
}

// Adam update of the FP32 master copy, re-rounding of the binary16
// parameters, and reset of the gradient accumulator.
__global__ void k_adam(float* __restrict__ master, __half* __restrict__ params, float* __restrict__ grad,
                       float* __restrict__ m1, float* __restrict__ m2, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kPropParams) return;
    const float g = grad[i];
    grad[i] = 0.0f;
    const float a = fmaf(0.9f, m1[i], 0.1f * g);
    const float b = fmaf(0.999f, m2[i], 0.001f * g * g);
    m1[i] = a;
    m2[i] = b;
    const float upd = lr * (a * c1) / (sqrtf(b * c2) + 1e-8f);
    master[i] -= upd;
    params[i] = __float2half_rn(master[i]);
}

egt_status launch_train(egt_proposal* p, const float* feats, const uint8_t* labels, int64_t m, int batch,
                        int sequential, float* loss_slot) {
    static bool attr_done[64] = {};
    if (!attr_done[p->device & 63]) {
        EGT_CUDA_TRY(cudaFuncSetAttribute(k_train_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
        attr_done[p->device & 63] = true;
    }
    TrainArgs t;
    t.params = p->params;
    t.feats = feats;
    t.labels = labels;
    t.m = m;
    t.batch = batch;
    t.seed = p->seed;
    t.step = p->step;
    t.sequential = sequential;
    t.grad = p->grad;
    t.loss = loss_slot;
    const unsigned G = (unsigned)((batch + kTB - 1) / kTB);
    k_train_batch<<<G, kTB, kTrainSmem, p->stream>>>(t);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

ProposeArgs propose_args(egt_handle* h) {
    ProposeArgs a{};
    a.p4 = h->p4;
    a.np = h->d_norm;
    for (int L = 0; L < kMaxLevels; L++) a.lv[L] = h->lv[L];
    a.n = (int)h->n;
    a.stride = 1;
    return a;
}

// Deterministic He-uniform initialisation (splitmix64 stream), biases zero.
void init_params(uint64_t seed, std::vector<float>& w) {
    w.assign(kPropParams, 0.0f);
    uint64_t st = seed;
    auto uni = [&]() {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t x = st;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        x ^= x >> 31;
        return (double)(x >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int rows, int cols) {
        const double lim = std::sqrt(6.0 / cols);
        for (int i = 0; i < rows * cols; i++) w[off + i] = (float)((2.0 * uni() - 1.0) * lim);
    };
    fill(kPW1, kPropHidden, kPropFeatures);
    fill(kPW2, kPropHidden, kPropHidden);
    fill(kPW3, kPropClasses, kPropHidden);
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

int proposal_k(const egt_proposal* p) { return p->k; }
int proposal_device(const egt_proposal* p) { return p->device; }

egt_status proposal_classes(egt_handle* h, const egt_proposal* p) {
    if (!h->pclass) EGT_CUDA_TRY(dev_alloc(h, &h->pclass, (size_t)h->n));
    ProposeArgs a = propose_args(h);
    a.params = p->params;
    a.tau = p->tau;
    a.cls = h->pclass;
    const unsigned T = 256, G = (unsigned)((h->n + T - 1) / T);
    k_propose<<<G, T, 0, h->stream>>>(a);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

}  // namespace egt

using namespace egt;

extern "C" {

egt_status egt_proposal_create(int device, int k, uint64_t seed, egt_proposal** out) {
    if (!out || k <= 0 || k > 255) { set_error("egt_proposal_create: bad argument (k in [1, 255])"); return EGT_ERR_ARG; }
    *out = nullptr;
    DeviceGuard g(device);
    auto* p = new egt_proposal();
    p->device = device;
    p->k = k;
    p->seed = seed;
    auto fail = [&](egt_status s) { egt_proposal_destroy(p); return s; };
    cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&p->params, sizeof(__half) * kPropParams);
    if (e == cudaSuccess) e = cudaMalloc(&p->master, sizeof(float) * kPropParams);
    if (e == cudaSuccess) e = cudaMalloc(&p->m1, sizeof(float) * kPropParams);
    if (e == cudaSuccess) e = cudaMalloc(&p->m2, sizeof(float) * kPropParams);
    if (e == cudaSuccess) e = cudaMalloc(&p->grad, sizeof(float) * kPropParams);
    if (e != cudaSuccess) {
        set_error(cuda_msg(e, "egt_proposal_create", __FILE__, __LINE__));
        return fail(e == cudaErrorMemoryAllocation ? EGT_ERR_NOMEM : EGT_ERR_CUDA);
    }
    std::vector<float> w;
    init_params(seed, w);
    std::vector<__half> hw(kPropParams);
    for (int i = 0; i < kPropParams; i++) {
        hw[i] = __float2half_rn(w[i]);
        w[i] = __half2float(hw[i]);  // master starts at the rounded values
    }
    e = cudaMemcpy(p->params, hw.data(), sizeof(__half) * kPropParams, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->master, w.data(), sizeof(float) * kPropParams, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(p->m1, 0, sizeof(float) * kPropParams);
    if (e == cudaSuccess) e = cudaMemset(p->m2, 0, sizeof(float) * kPropParams);
    if (e == cudaSuccess) e = cudaMemset(p->grad, 0, sizeof(float) * kPropParams);
    if (e != cudaSuccess) {
        set_error(cuda_msg(e, "egt_proposal_create", __FILE__, __LINE__));
        return fail(EGT_ERR_CUDA);
    }
    *out = p;
    return EGT_OK;
}

void egt_proposal_destroy(egt_proposal* p) {
    if (!p) return;
    DeviceGuard g(p->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    cudaFree(p->params);
    cudaFree(p->master);
    cudaFree(p->m1);
    cudaFree(p->m2);
    cudaFree(p->grad);
    cudaFree(p->loss);
    cudaFree(p->feats);
    cudaFree(p->labels);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
}

egt_status egt_proposal_collect(egt_proposal* p, egt_handle* h, int stride) {
    if (!p || !h || stride < 1) { set_error("egt_proposal_collect: bad argument"); return EGT_ERR_ARG; }
    if (!h->kth || h->k != p->k || h->is_mesh) {
        set_error("egt_proposal_collect: the handle needs a grid kNN with the proposal's k");
        return EGT_ERR_STATE;
    }
    if (h->cfg.device != p->device) { set_error("egt_proposal_collect: proposal on another device"); return EGT_ERR_ARG; }
    DeviceGuard g(p->device);
    const int64_t rows = (h->n + stride - 1) / stride;
    if (p->m + rows > p->cap) {
        const int64_t cap = std::max<int64_t>(p->m + rows, p->cap * 2);
        float* nf = nullptr;
        uint8_t* nl = nullptr;
        EGT_CUDA_TRY(cudaStreamSynchronize(h->stream));
        EGT_CUDA_TRY(cudaStreamSynchronize(p->stream));
        EGT_CUDA_TRY(cudaMalloc(&nf, sizeof(float) * kPropFeatures * cap));
        EGT_CUDA_TRY(cudaMalloc(&nl, (size_t)cap));
        if (p->m) {
            EGT_CUDA_TRY(cudaMemcpy(nf, p->feats, sizeof(float) * kPropFeatures * p->m, cudaMemcpyDeviceToDevice));
            EGT_CUDA_TRY(cudaMemcpy(nl, p->labels, (size_t)p->m, cudaMemcpyDeviceToDevice));
        }
        cudaFree(p->feats);
        cudaFree(p->labels);
        p->feats = nf;
        p->labels = nl;
        p->cap = cap;
    }
    ProposeArgs a = propose_args(h);
    a.stride = stride;
    a.feats = p->feats + p->m * kPropFeatures;
    a.kth = h->kth;
    a.labels = p->labels + p->m;
    const unsigned T = 256, G = (unsigned)((rows + T - 1) / T);
    k_propose<<<G, T, 0, h->stream>>>(a);
    EGT_LAUNCH_CHECK();
    EGT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    p->m += rows;
    return EGT_OK;
}

int64_t egt_proposal_samples(const egt_proposal* p) { return p ? p->m : 0; }

egt_status egt_proposal_train(egt_proposal* p, int steps, int batch, float lr, float* loss_out) {
    if (!p || steps < 0 || batch < 1 || !(lr > 0.0f)) { set_error("egt_proposal_train: bad argument"); return EGT_ERR_ARG; }
    if (p->m == 0) { set_error("egt_proposal_train: no training samples collected"); return EGT_ERR_STATE; }
    DeviceGuard g(p->device);
    if (steps > p->loss_cap) {
        cudaFree(p->loss);
        p->loss = nullptr;
        EGT_CUDA_TRY(cudaMalloc(&p->loss, sizeof(float) * steps));
        p->loss_cap = steps;
    }
    if (steps) EGT_CUDA_TRY(cudaMemsetAsync(p->loss, 0, sizeof(float) * steps, p->stream));
    for (int s = 0; s < steps; s++) {
        EGT_TRY(launch_train(p, p->feats, p->labels, p->m, batch, 0, p->loss + s));
        p->step++;
        const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, (double)p->step)));
        const float c2 = (float)(1.0 / (1.0 - std::pow(0.999, (double)p->step)));
        k_adam<<<(kPropParams + 255) / 256, 256, 0, p->stream>>>(p->master, p->params, p->grad, p->m1, p->m2, lr,
                                                                  c1, c2);
        EGT_LAUNCH_CHECK();
    }
    if (loss_out && steps)
        EGT_CUDA_TRY(cudaMemcpyAsync(loss_out, p->loss, sizeof(float) * steps, cudaMemcpyDeviceToHost, p->stream));
    EGT_CUDA_TRY(cudaStreamSynchronize(p->stream));
    return EGT_OK;
}

egt_status egt_proposal_gradients(egt_proposal* p, const float* feats, const uint8_t* labels, int m, float* grads,
                                  float* loss) {
    if (!p || !feats || !labels || !grads || m < 1) { set_error("egt_proposal_gradients: bad argument"); return EGT_ERR_ARG; }
    DeviceGuard g(p->device);
    float* df = nullptr;
    uint8_t* dl = nullptr;
    float* dloss = nullptr;
    EGT_CUDA_TRY(cudaMalloc(&df, sizeof(float) * kPropFeatures * m));
    cudaError_t e = cudaMalloc(&dl, (size_t)m);
    if (e == cudaSuccess) e = cudaMalloc(&dloss, sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(df, feats, sizeof(float) * kPropFeatures * m, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dl, labels, (size_t)m, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dloss, 0, sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(p->grad, 0, sizeof(float) * kPropParams);
    egt_status st = EGT_OK;
    if (e != cudaSuccess) {
        set_error(cuda_msg(e, "egt_proposal_gradients", __FILE__, __LINE__));
        st = EGT_ERR_CUDA;
    }
    if (st == EGT_OK) st = launch_train(p, df, dl, m, m, 1, dloss);
    if (st == EGT_OK) {
        e = cudaStreamSynchronize(p->stream);
        if (e == cudaSuccess) e = cudaMemcpy(grads, p->grad, sizeof(float) * kPropParams, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && loss) e = cudaMemcpy(loss, dloss, sizeof(float), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemset(p->grad, 0, sizeof(float) * kPropParams);
        if (e != cudaSuccess) {
            set_error(cuda_msg(e, "egt_proposal_gradients", __FILE__, __LINE__));
            st = EGT_ERR_CUDA;
        }
    }
    cudaFree(df);
    cudaFree(dl);
    cudaFree(dloss);
    return st;
}

egt_status egt_proposal_get_params(const egt_proposal* p, uint16_t* params) {
    if (!p || !params) { set_error("egt_proposal_get_params: bad argument"); return EGT_ERR_ARG; }
    DeviceGuard g(p->device);
    EGT_CUDA_TRY(cudaStreamSynchronize(p->stream));
    EGT_CUDA_TRY(cudaMemcpy(params, p->params, sizeof(__half) * kPropParams, cudaMemcpyDeviceToHost));
    return EGT_OK;
}

egt_status egt_proposal_set_params(egt_proposal* p, const uint16_t* params) {
    if (!p || !params) { set_error("egt_proposal_set_params: bad argument"); return EGT_ERR_ARG; }
    DeviceGuard g(p->device);
    std::vector<float> w(kPropParams);
    const __half* hp = reinterpret_cast<const __half*>(params);
    for (int i = 0; i < kPropParams; i++) w[i] = __half2float(hp[i]);
    EGT_CUDA_TRY(cudaStreamSynchronize(p->stream));
    EGT_CUDA_TRY(cudaMemcpy(p->params, params, sizeof(__half) * kPropParams, cudaMemcpyHostToDevice));
    EGT_CUDA_TRY(cudaMemcpy(p->master, w.data(), sizeof(float) * kPropParams, cudaMemcpyHostToDevice));
    EGT_CUDA_TRY(cudaMemset(p->m1, 0, sizeof(float) * kPropParams));
    EGT_CUDA_TRY(cudaMemset(p->m2, 0, sizeof(float) * kPropParams));
    p->step = 0;
    return EGT_OK;
}

egt_status egt_proposal_set_tau(egt_proposal* p, float tau) {
    if (!p || !(tau > 0.0f && tau <= 1.0f)) { set_error("egt_proposal_set_tau: tau must be in (0, 1]"); return EGT_ERR_ARG; }
    p->tau = tau;
    return EGT_OK;
}

float egt_proposal_get_tau(const egt_proposal* p) { return p ? p->tau : 0.0f; }

egt_status egt_proposal_tune(egt_proposal* p, egt_handle* h, const float* taus, int ntau, float* ms_out) {
    if (!p || !h || !taus || ntau < 1) { set_error("egt_proposal_tune: bad argument"); return EGT_ERR_ARG; }
    if (h->k != p->k) { set_error("egt_proposal_tune: the handle's k differs from the proposal's"); return EGT_ERR_STATE; }
    if (h->cfg.device != p->device) { set_error("egt_proposal_tune: proposal on another device"); return EGT_ERR_ARG; }
    DeviceGuard g(p->device);
    h->last_knn_learned = true;
    for (int i = 0; i < ntau; i++)
        if (!(taus[i] > 0.0f && taus[i] <= 1.0f)) { set_error("egt_proposal_tune: tau must be in (0, 1]"); return EGT_ERR_ARG; }
    const float keep = p->tau;
    float best = 1e30f, best_tau = keep;
    for (int i = 0; i < ntau; i++) {
        p->tau = taus[i];
        EGT_TRY(run_knn_learned(h, p->k, p));  // warm
        EGT_TRY(run_knn_learned(h, p->k, p));
        EGT_CUDA_TRY(cudaEventSynchronize(h->ev[3]));
        const float ms = elapsed_ms(h->ev[2], h->ev[3]);
        if (ms_out) ms_out[i] = ms;
        if (ms < best) { best = ms; best_tau = taus[i]; }
    }
    p->tau = best_tau;
    return EGT_OK;
}

egt_status egt_proposal_inspect(const egt_proposal* p, egt_handle* h, float* feats, uint8_t* labels,
                                uint8_t* classes) {
    if (!p || !h) { set_error("egt_proposal_inspect: bad argument"); return EGT_ERR_ARG; }
    if (labels && (!h->kth || h->k != p->k)) {
        set_error("egt_proposal_inspect: labels need a grid kNN with the proposal's k");
        return EGT_ERR_STATE;
    }
    if (h->cfg.device != p->device) { set_error("egt_proposal_inspect: proposal on another device"); return EGT_ERR_ARG; }
    DeviceGuard g(p->device);
    const int64_t n = h->n;
    float* df = nullptr;
    uint8_t* dl = nullptr;
    if (feats) EGT_CUDA_TRY(dev_alloc(h, &df, sizeof(float) * kPropFeatures * n));
    if (labels) EGT_CUDA_TRY(dev_alloc(h, &dl, (size_t)n));
    if (feats || labels) {
        ProposeArgs a = propose_args(h);
        a.feats = df;
        a.kth = h->kth;
        a.labels = dl;
        const unsigned T = 256, G = (unsigned)((n + T - 1) / T);
        k_propose<<<G, T, 0, h->stream>>>(a);
        EGT_LAUNCH_CHECK();
    }
    if (classes) EGT_TRY(proposal_classes(h, p));
    if (feats)
        EGT_CUDA_TRY(cudaMemcpyAsync(feats, df, sizeof(float) * kPropFeatures * n, cudaMemcpyDeviceToHost, h->stream));
    if (labels) EGT_CUDA_TRY(cudaMemcpyAsync(labels, dl, (size_t)n, cudaMemcpyDeviceToHost, h->stream));
    if (classes) EGT_CUDA_TRY(cudaMemcpyAsync(classes, h->pclass, (size_t)n, cudaMemcpyDeviceToHost, h->stream));
    dev_free(h, df);
    dev_free(h, dl);
    EGT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return EGT_OK;
}

}  // extern "C"
