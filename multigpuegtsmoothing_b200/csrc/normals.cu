// Unoriented PCA normals.
//
// Reference: calculateNormal (Normal_CUDA.cu:87-144): centroid over the point
// and its (EGT-filtered) neighbours, covariance over the neighbours only, then
// the iterative symmetric 3x3 eigensolver (EigenSolver.cuh:124-392, the
// Householder + Givens algorithm of D. Eberly, "A Robust Eigensolver for 3x3
// Symmetric Matrices", Geometric Tools) with sortType = +1; the normal is the
// eigenvector of the smallest eigenvalue, normalised.
//
// FP32 path: same operation order and fused multiply-adds as the reference
// build, so the normal (and its raw sign, which seeds the orientation) is the
// reference's.  FP64 path: when the gap between the two smallest eigenvalues is
// below gap_tol times the largest, the covariance and the eigensolve are
// redone in double precision (FP32 error grows as 1/gap there).
#include "egt_internal.cuh"

namespace egt {
namespace {

template <typename T> struct Ops;
template <> struct Ops<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float sqrt_(float a) { return __fsqrt_rn(a); }
    static __device__ __forceinline__ float lin_add(float c, float a, float s, float b) { return fs_lin2_add(c, a, s, b); }
    static __device__ __forceinline__ float lin_sub(float s, float a, float c, float b) { return fs_lin2_sub(s, a, c, b); }
    static __device__ __forceinline__ float hyp2(float u, float v) { return fs_sq2(u, v); }
    static __device__ __forceinline__ int exponent(float v) { int e; frexpf(v, &e); return e; }
    static constexpr int kAlpha = 149;
};
template <> struct Ops<double> {
    static __device__ __forceinline__ double add(double a, double b) { return a + b; }
    static __device__ __forceinline__ double sub(double a, double b) { return a - b; }
    static __device__ __forceinline__ double mul(double a, double b) { return a * b; }
    static __device__ __forceinline__ double div(double a, double b) { return a / b; }
    static __device__ __forceinline__ double sqrt_(double a) { return sqrt(a); }
    static __device__ __forceinline__ double lin_add(double c, double a, double s, double b) { return fma(c, a, s * b); }
    static __device__ __forceinline__ double lin_sub(double s, double a, double c, double b) { return fma(s, a, -(c * b)); }
    static __device__ __forceinline__ double hyp2(double u, double v) { return fma(u, u, v * v); }
    static __device__ __forceinline__ int exponent(double v) { int e; frexp(v, &e); return e; }
    static constexpr int kAlpha = 1074;
};

template <typename T>
__device__ __forceinline__ void cos_sin(T u, T v, T& c, T& s) {  // EigenSolver.cuh:353-373
    using O = Ops<T>;
    const T len = O::sqrt_(O::hyp2(u, v));
    if (len > T(0)) {
        c = O::div(u, len);
        s = O::div(v, len);
        if (c > T(0)) { c = -c; s = -s; }
    } else {
        c = T(-1);
        s = T(0);
    }
}

template <typename T>
__device__ __forceinline__ bool converged(T d0, T d1, T sd) {  // EigenSolver.cuh:375-391 (non-aggressive)
    using O = Ops<T>;
    const T sum = O::add(fabs(d0), fabs(d1));
    return O::add(sum, fabs(sd)) == sum;
}

// Returns eigenvalues ascending in ev[] and the eigenvector of ev[0] in n[].
template <typename T>
__device__ void eigen_smallest(T a00, T a01, T a02, T a11, T a12, T a22, T ev[3], T n[3]) {
    using O = Ops<T>;
    const T half = T(0.5), one = T(1);
    bool rot = false;
    T c = 0, s = 0;
    cos_sin<T>(a12, -a02, c, s);
    T t0 = O::lin_add(c, a00, s, a01);
    T t1 = O::lin_add(c, a01, s, a11);
    T t2 = O::lin_sub(s, a00, c, a01);
    T t3 = O::lin_sub(s, a01, c, a11);
    T b00 = O::lin_add(c, t0, s, t1);
    T b01 = O::lin_sub(s, t0, c, t1);
    T b11 = O::lin_sub(s, t2, c, t3);
    T b12 = O::lin_sub(s, a02, c, a12);
    T b22 = a22;
    T Q[3][3] = {{c, s, T(0)}, {s, -c, T(0)}, {T(0), T(0), T(1)}};
    T c2 = 0, s2 = 0;
    if (fabs(b12) <= fabs(b01)) {
        const int imax = 2 * (O::exponent(b12) + O::kAlpha + 1);
        for (int i = 0; i < imax; ++i) {
            cos_sin<T>(O::mul(half, O::sub(b00, b11)), b01, c2, s2);
            s = O::sqrt_(O::mul(half, O::sub(one, c2)));
            c = O::div(O::mul(half, s2), s);
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const T u0 = O::lin_add(c, Q[r][0], s, Q[r][1]);
                const T u1 = Q[r][2];
                const T u2 = O::lin_sub(c, Q[r][1], s, Q[r][0]);
                Q[r][0] = u0; Q[r][1] = u1; Q[r][2] = u2;
            }
            rot = !rot;
            t0 = O::lin_add(c, b00, s, b01);
            t1 = O::lin_add(c, b01, s, b11);
            t2 = O::lin_sub(s, b00, c, b01);
            t3 = O::lin_sub(s, b01, c, b11);
            b00 = O::lin_add(c, t0, s, t1);
            b01 = O::mul(s, b12);
            b11 = b22;
            b12 = O::mul(c, b12);
            b22 = O::lin_sub(s, t2, c, t3);
            if (converged<T>(b00, b11, b01)) {
                cos_sin<T>(O::mul(half, O::sub(b00, b11)), b01, c2, s2);
                s = O::sqrt_(O::mul(half, O::sub(one, c2)));
                c = O::div(O::mul(half, s2), s);
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    const T u0 = O::lin_add(c, Q[r][0], s, Q[r][1]);
                    const T u1 = O::lin_sub(s, Q[r][0], c, Q[r][1]);
                    Q[r][0] = u0; Q[r][1] = u1;
                }
                rot = !rot;
                t0 = O::lin_add(c, b00, s, b01);
                t1 = O::lin_add(c, b01, s, b11);
                t2 = O::lin_sub(s, b00, c, b01);
                t3 = O::lin_sub(s, b01, c, b11);
                b00 = O::lin_add(c, t0, s, t1);
                b11 = O::lin_sub(s, t2, c, t3);
                break;
            }
        }
    } else {
        const int imax = 2 * (O::exponent(b01) + O::kAlpha + 1);
        for (int i = 0; i < imax; ++i) {
            cos_sin<T>(O::mul(half, O::sub(b11, b22)), b12, c2, s2);
            s = O::sqrt_(O::mul(half, O::sub(one, c2)));
            c = O::div(O::mul(half, s2), s);
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const T u0 = O::lin_add(c, Q[r][1], s, Q[r][2]);
                const T u1 = Q[r][0];
                const T u2 = O::lin_sub(c, Q[r][2], s, Q[r][1]);
                Q[r][0] = u0; Q[r][1] = u1; Q[r][2] = u2;
            }
            rot = !rot;
            t0 = O::lin_add(c, b11, s, b12);
            t1 = O::lin_add(c, b12, s, b22);
            t2 = O::lin_sub(s, b11, c, b12);
            t3 = O::lin_sub(s, b12, c, b22);
            b22 = O::lin_sub(s, t2, c, t3);
            b12 = O::mul(-s, b01);
            b11 = b00;
            b01 = O::mul(c, b01);
            b00 = O::lin_add(c, t0, s, t1);
            if (converged<T>(b11, b22, b12)) {
                cos_sin<T>(O::mul(half, O::sub(b11, b22)), b12, c2, s2);
                s = O::sqrt_(O::mul(half, O::sub(one, c2)));
                c = O::div(O::mul(half, s2), s);
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    const T u0 = O::lin_add(c, Q[r][1], s, Q[r][2]);
                    const T u1 = O::lin_sub(s, Q[r][1], c, Q[r][2]);
                    Q[r][1] = u0; Q[r][2] = u1;
                }
                rot = !rot;
                t0 = O::lin_add(c, b11, s, b12);
                t1 = O::lin_add(c, b12, s, b22);
                t2 = O::lin_sub(s, b11, c, b12);
                t3 = O::lin_sub(s, b12, c, b22);
                b11 = O::lin_add(c, t0, s, t1);
                b22 = O::lin_sub(s, t2, c, t3);
                break;
            }
        }
    }
    // SortEigenstuff, increasing (EigenSolver.cuh:29-122); column j of Q is eigenvector j
    const T e[3] = {b00, b11, b22};
    int i0, i1, i2;
    if (e[0] < e[1]) {
        if (e[2] < e[0]) { i0 = 2; i1 = 0; i2 = 1; }
        else if (e[2] < e[1]) { i0 = 0; i1 = 2; i2 = 1; rot = !rot; }
        else { i0 = 0; i1 = 1; i2 = 2; }
    } else {
        if (e[2] < e[1]) { i0 = 2; i1 = 1; i2 = 0; rot = !rot; }
        else if (e[2] < e[0]) { i0 = 1; i1 = 2; i2 = 0; }
        else { i0 = 1; i1 = 0; i2 = 2; rot = !rot; }
    }
    (void)rot;  // only flips evec[2]; the normal is evec[0]
    ev[0] = e[i0]; ev[1] = e[i1]; ev[2] = e[i2];
    n[0] = Q[0][i0]; n[1] = Q[1][i0]; n[2] = Q[2][i0];
}

__global__ void __launch_bounds__(128) k_normals(const float4* __restrict__ p4, const int* __restrict__ off,
                                                 const int* __restrict__ col, int n, float gap_tol,
                                                 float* __restrict__ nrm, unsigned long long* __restrict__ nfb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = p4[i];
    const int e0 = off[i], e1 = off[i + 1];
    float sx = p.x, sy = p.y, sz = p.z;
    for (int e = e0; e < e1; e++) {
        const float4 q = p4[col[e]];
        sx = __fadd_rn(sx, q.x); sy = __fadd_rn(sy, q.y); sz = __fadd_rn(sz, q.z);
    }
    const float cnt = (float)(1 + e1 - e0);
    const float mx = __fdiv_rn(sx, cnt), my = __fdiv_rn(sy, cnt), mz = __fdiv_rn(sz, cnt);
    float c00 = 0, c01 = 0, c02 = 0, c11 = 0, c12 = 0, c22 = 0;
    for (int e = e0; e < e1; e++) {
        const float4 q = p4[col[e]];
        const float dx = __fsub_rn(q.x, mx), dy = __fsub_rn(q.y, my), dz = __fsub_rn(q.z, mz);
        c00 = __fmaf_rn(dx, dx, c00); c01 = __fmaf_rn(dx, dy, c01); c02 = __fmaf_rn(dx, dz, c02);
        c11 = __fmaf_rn(dy, dy, c11); c12 = __fmaf_rn(dy, dz, c12); c22 = __fmaf_rn(dz, dz, c22);
    }
    float ev[3], v[3];
    eigen_smallest<float>(c00, c01, c02, c11, c12, c22, ev, v);
    float ox, oy, oz;
    if (gap_tol > 0.f && (ev[1] - ev[0]) < gap_tol * fabsf(ev[2])) {
        // near-degenerate smallest pair: redo in double precision
        double dx0 = p.x, dy0 = p.y, dz0 = p.z;
        for (int e = e0; e < e1; e++) {
            const float4 q = p4[col[e]];
            dx0 += q.x; dy0 += q.y; dz0 += q.z;
        }
        const double dc = (double)(1 + e1 - e0);
        const double gx = dx0 / dc, gy = dy0 / dc, gz = dz0 / dc;
        double d00 = 0, d01 = 0, d02 = 0, d11 = 0, d12 = 0, d22 = 0;
        for (int e = e0; e < e1; e++) {
            const float4 q = p4[col[e]];
            const double ax = q.x - gx, ay = q.y - gy, az = q.z - gz;
            d00 += ax * ax; d01 += ax * ay; d02 += ax * az; d11 += ay * ay; d12 += ay * az; d22 += az * az;
        }
        double dev[3], dv[3];
        eigen_smallest<double>(d00, d01, d02, d11, d12, d22, dev, dv);
        const double l = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
        ox = (float)(dv[0] / l); oy = (float)(dv[1] / l); oz = (float)(dv[2] / l);
        atomicAdd(nfb, 1ull);
    } else {
        const float l = __fsqrt_rn(fs_sq3(v[0], v[1], v[2]));
        ox = __fdiv_rn(v[0], l); oy = __fdiv_rn(v[1], l); oz = __fdiv_rn(v[2], l);
    }
    nrm[i] = ox;
    nrm[n + i] = oy;
    nrm[2 * (size_t)n + i] = oz;
}

}  // namespace

egt_status run_normals(egt_handle* h) {
    EGT_TRY(ensure_csr(h));
    const int n = (int)h->n;
    if (!h->nrm) EGT_CUDA_TRY(dev_alloc(h, &h->nrm, sizeof(float) * 3 * (size_t)n));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrNormFallback, 0, sizeof(unsigned long long), h->stream));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[8], h->stream));
    k_normals<<<(unsigned)((n + 127) / 128), 128, 0, h->stream>>>(h->p4, h->csr_off, h->csr_col, n,
                                                                   h->cfg.normals_gap_tol, h->nrm,
                                                                   h->d_counters + kCtrNormFallback);
    EGT_LAUNCH_CHECK();
    EGT_CUDA_TRY(cudaEventRecord(h->ev[9], h->stream));
    return EGT_OK;
}

}  // namespace egt
