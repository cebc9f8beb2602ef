// Taubin smoothing without any device allocation.
//
// Some callers cannot allocate device memory themselves:
//   * hosts that hand all of their GPU memory to one allocator of their own
//     (a caching allocator or a pre-sized arena) and forbid other
//     allocations, where a cudaMalloc can fail or fragment that memory;
//   * real-time loops (a scanner's or a robot's per-frame smoothing) where
//     the implicit device synchronisation of cudaMalloc/cudaFree stalls the
//     loop.
// egt_taubin_noalloc serves them: the caller passes the input and output
// positions and the neighbourhood CSR, and the only intermediate buffer the
// smoothing needs -- the positions between the lambda and the mu half-step --
// lives in the fixed array below.
//
// When the memory is committed: CUDA loads a library's kernel modules, and
// with them their __device__ arrays, lazily -- on a device's first use of
// them -- unless CUDA_MODULE_LOADING=EAGER asks for it at context creation.
// Every call therefore starts with a set-up step on the current device that
// resolves the array's device address (cudaGetSymbolAddress) and loads the
// half-step kernel's module (cudaFuncGetAttributes), whatever `iters` is.  On
// the first call on a device this commits the 16 MB array and the module;
// later calls only look both up.  Make that first call before any stream
// capture and at a point where the device can still take a 16 MB commitment.
// Resolving the address on every call (a table lookup once loaded) also keeps
// it right after cudaDeviceReset, which unloads the module.
//
// Limits and sharing rules:
//   * at most kNoAllocMaxPoints points (larger inputs are rejected);
//   * a device holds the 16 MB array from its first call until the process
//     exits;
//   * all calls share the one array: calls that may overlap on the GPU (on
//     different streams, or from several host threads) race with each other
//     and must be serialised by the caller;
//   * the array keeps the previous call's contents; nothing in it needs to
//     start at zero, because every half-step writes all n entries before the
//     next one reads them.
#include "egt_internal.cuh"

namespace egt {
egt_status taubin_preload();
egt_status taubin_launch(const float4* pin, float4* pout, const int* off, const int* col, int n, float scale,
                         cudaStream_t st);
}

namespace {

constexpr int64_t kNoAllocMaxPoints = int64_t(1) << 20;  // 16 MB of float4

static __device__ __align__(256) float4 g_noalloc_scratch[kNoAllocMaxPoints];

// Set-up on the current device: the device address of g_noalloc_scratch (in
// host code the array's name is only a host-side stand-in, which a kernel
// must never be given) and the half-step kernel's module.
egt_status noalloc_setup(float4** out) {
    void* p = nullptr;
    EGT_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    EGT_TRY(egt::taubin_preload());
    *out = static_cast<float4*>(p);
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
    EGT_TRY(noalloc_setup(&scratch));
    cudaStream_t st = (cudaStream_t)stream;
    const float4* in = reinterpret_cast<const float4*>(pos_in);
    float4* out = reinterpret_cast<float4*>(pos_out);
    if (iters == 0) {
        if (in != out)
            EGT_CUDA_TRY(cudaMemcpyAsync(out, in, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToDevice, st));
        return EGT_OK;
    }
    for (int it = 0; it < iters; it++) {
        EGT_TRY(egt::taubin_launch(it == 0 ? in : out, scratch, csr_off, csr_col, (int)n, lambda, st));
        EGT_TRY(egt::taubin_launch(scratch, out, csr_off, csr_col, (int)n, mu, st));
    }
    return EGT_OK;
}
