// Taubin smoothing without any device allocation.
//
// Some callers cannot allocate device memory themselves: hosts that hand all
// of their GPU memory to one allocator of their own and forbid other
// allocations, real-time loops where the implicit synchronisation of
// cudaMalloc/cudaFree is not acceptable, and code that records its work into
// a CUDA graph, where an allocation inside the recorded region is not allowed.
// egt_taubin_noalloc serves them: the caller passes the input and output
// positions and the neighbourhood CSR, and the only intermediate buffer the
// smoothing needs -- the positions between the lambda and the mu half-step --
// lives in the fixed array below, reserved once per GPU when the library is
// loaded.
//
// Limits and sharing rules:
//   * at most kNoAllocMaxPoints points (larger inputs are rejected);
//   * every GPU that loads the library holds the 16 MB array until the process
//     exits;
//   * all calls share the one array: calls that may overlap on the GPU (on
//     different streams, or from several host threads) race with each other
//     and must be serialised by the caller;
//   * the array keeps the previous call's contents; nothing in it needs to
//     start at zero, because every half-step writes all n entries before the
//     next one reads them.
#include <mutex>
#include "egt_internal.cuh"

namespace egt {
egt_status taubin_launch(const float4* pin, float4* pout, const int* off, const int* col, int n, float scale,
                         cudaStream_t st);
}

namespace {

constexpr int64_t kNoAllocMaxPoints = int64_t(1) << 20;  // 16 MB of float4

static __device__ __align__(256) float4 g_noalloc_scratch[kNoAllocMaxPoints];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
float4* g_scratch_ptr[kMaxDevices] = {};

// Resolves the device address of g_noalloc_scratch on the current device, once
// per device.  In host code the array's name is only a host-side stand-in:
// passing it to a kernel directly would fault or use the wrong memory.
egt_status scratch_for_current_device(float4** out) {
    int dev = 0;
    EGT_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        egt::set_error("egt_taubin_noalloc: device ordinal out of range");
        return EGT_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        EGT_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_ptr[dev] = static_cast<float4*>(p);
    }
    *out = g_scratch_ptr[dev];
    return EGT_OK;
}

}  // namespace

extern "C" egt_status egt_taubin_noalloc(const float* pos_in, float* pos_out, const int* csr_off,
                                         const int* csr_col, int64_t n, int iters, float lambda, float mu,
                                         void* stream) {
    if (!pos_in || !pos_out || !csr_off || (!csr_col && n > 0)) {
        egt::set_error("egt_taubin_noalloc: null pointer argument");
        return EGT_ERR_ARG;
    }
    if (n < 1 || iters < 0) {
        egt::set_error("egt_taubin_noalloc: need n >= 1 and iters >= 0");
        return EGT_ERR_ARG;
    }
    if (n > kNoAllocMaxPoints) {
        egt::set_error("egt_taubin_noalloc: n exceeds the fixed scratch capacity of 1048576 points");
        return EGT_ERR_ARG;
    }
    float4* scratch = nullptr;
    EGT_TRY(scratch_for_current_device(&scratch));
    cudaStream_t st = (cudaStream_t)stream;
    const float4* in = reinterpret_cast<const float4*>(pos_in);
    float4* out = reinterpret_cast<float4*>(pos_out);
    if (iters == 0) {
        EGT_CUDA_TRY(cudaMemcpyAsync(out, in, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToDevice, st));
        return EGT_OK;
    }
    for (int it = 0; it < iters; it++) {
        EGT_TRY(egt::taubin_launch(it == 0 ? in : out, scratch, csr_off, csr_col, (int)n, lambda, st));
        EGT_TRY(egt::taubin_launch(scratch, out, csr_off, csr_col, (int)n, mu, st));
    }
    return EGT_OK;
}
