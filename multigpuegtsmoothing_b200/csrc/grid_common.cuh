// Device helpers of the grid build shared by the single-cloud (grid.cu) and
// batched (batch.cu) builds.
#pragma once
#include "egt_internal.cuh"

namespace egt {

// Order-preserving float <-> uint32 maps for atomic min/max of floats.
__device__ __forceinline__ uint32_t f2ord(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Scalar cube of InitStructure: thrust::reduce(.., 1e8f, minimum) - 1e-6f and
// thrust::reduce(.., -1e8f, maximum) + 1e-6f per axis, then min/max over axes.
__device__ __forceinline__ NormParams finalize_norm(const uint32_t* acc, float eps, float thres0, int64_t n) {
    float lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        lo[d] = __fsub_rn(fminf(1e8f, ord2f(acc[d])), 1e-6f);
        hi[d] = __fadd_rn(fmaxf(-1e8f, ord2f(acc[3 + d])), 1e-6f);
    }
    float mn = lo[0], mx = hi[0];
    // std::min / std::max semantics (returns the first argument on ties)
    mn = (lo[1] < mn) ? lo[1] : mn;
    mn = (lo[2] < mn) ? lo[2] : mn;
    mx = (mx < hi[1]) ? hi[1] : mx;
    mx = (mx < hi[2]) ? hi[2] : mx;
    NormParams p;
    p.mn = mn;
    p.mx = mx;
    p.a = -eps;
    p.b = (float)(1.0 + (double)eps);
    float t = thres0;
    t = __fdiv_rn(t, __fsub_rn(mx, mn));
    t = __fmul_rn(t, t);
    p.thres = t;
    p.n = (int)n;
    return p;
}

}  // namespace egt
