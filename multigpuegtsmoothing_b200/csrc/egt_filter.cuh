// Elliptic-Gabriel filter of one query's list (one warp), shared by the
// single-cloud (egt.cu) and batched (batch.cu) kernels.  See egt.cu for the
// reference correspondence.  Returns the number of kept entries (uniform);
// dropped entries of `row` are set to -1.  tests counts the ellipsoid tests
// this lane evaluated.
#pragma once
#include "egt_internal.cuh"

namespace egt {
namespace {

template <int S>
__device__ __forceinline__ int egt_query(const float4* __restrict__ p4, float4 p, int* __restrict__ row, int k,
                                         float alpha, int lane, unsigned& tests) {
    int nb[S];
    float4 v[S];
    bool keep[S], test[S];
    float ax[S], ay[S], az[S], px[S], py[S], pz[S], qx[S], qy[S], qz[S], tx[S], ty[S], tz[S], dd[S];
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        nb[s] = t < k ? row[t] : -1;
        v[s] = nb[s] >= 0 ? p4[nb[s]] : make_float4(0.f, 0.f, 0.f, 0.f);
        keep[s] = nb[s] != -1;
        test[s] = false;
        if (keep[s]) {
            const float xi = v[s].x, yi = v[s].y, zi = v[s].z;
            const float xo = __fmul_rn(0.5f, __fadd_rn(xi, p.x));
            const float yo = __fmul_rn(0.5f, __fadd_rn(yi, p.y));
            const float zo = __fmul_rn(0.5f, __fadd_rn(zi, p.z));
            const float d = __fdiv_rn(__fsqrt_rn(fs_dist3(xi, yi, zi, p.x, p.y, p.z)), 2.0f);
            float ex = __fsub_rn(xi, p.x), ey = __fsub_rn(yi, p.y), ez = __fsub_rn(zi, p.z);
            const float len = __fsqrt_rn(fs_sq3(ex, ey, ez));
            if (!((double)d < 1e-6) && !((double)len < 1e-6)) {
                test[s] = true;
                // x axis
                ex = __fdiv_rn(ex, len); ey = __fdiv_rn(ey, len); ez = __fdiv_rn(ez, len);
                // y axis: unit vector perpendicular to x (EGT_CUDA.cu:61-95)
                float m = fabsf(ex);
                int ci = 0;
                if (m < fabsf(ey)) { ci = 1; m = fabsf(ey); }
                if (m < fabsf(ez)) ci = 2;
                float ux = 1.0f, uy = 1.0f, uz = 1.0f;
                if (ci == 0) ux = __fdiv_rn(__fsub_rn(-ey, ez), ex);
                else if (ci == 1) uy = __fdiv_rn(__fsub_rn(-ex, ez), ey);
                else uz = __fdiv_rn(__fsub_rn(-ex, ey), ez);
                const float ul = __fsqrt_rn(fs_sq3(ux, uy, uz));
                ux = __fdiv_rn(ux, ul); uy = __fdiv_rn(uy, ul); uz = __fdiv_rn(uz, ul);
                // z axis = x cross y, normalised
                float wx = fs_cross1(ey, uz, uy, ez);
                float wy = fs_cross1(ux, ez, ex, uz);
                float wz = fs_cross1(ex, uy, ux, ey);
                const float wl = __fsqrt_rn(fs_sq3(wx, wy, wz));
                wx = __fdiv_rn(wx, wl); wy = __fdiv_rn(wy, wl); wz = __fdiv_rn(wz, wl);
                ax[s] = ex; ay[s] = ey; az[s] = ez;
                px[s] = ux; py[s] = uy; pz[s] = uz;
                qx[s] = wx; qy[s] = wy; qz[s] = wz;
                tx[s] = -fs_affine(ex, ey, ez, 0.0f, xo, yo, zo);
                ty[s] = -fs_affine(ux, uy, uz, 0.0f, xo, yo, zo);
                tz[s] = -fs_affine(wx, wy, wz, 0.0f, xo, yo, zo);
                dd[s] = __fmul_rn(d, d);
            }
        }
    }
    const float aa = __fmul_rn(alpha, alpha);
    const float inv_aa = 1.0f / aa;
    // last slot index that still has something to test
    int hi = -1;
#pragma unroll
    for (int s = 0; s < S; s++)
        if (test[s]) hi = lane + 32 * s;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    for (int jp = 0; jp < hi; jp++) {
        if ((jp & 7) == 0) {  // stop once every slot with a pending test is decided
            bool pending = false;
#pragma unroll
            for (int s = 0; s < S; s++) pending |= test[s] && keep[s] && jp < lane + 32 * s;
            if (!__any_sync(0xffffffffu, pending)) break;
        }
        const int sl = jp & 31, ss = jp >> 5;
        int bn = nb[0];
        float4 bv = v[0];
#pragma unroll
        for (int s = 1; s < S; s++)
            if (ss == s) { bn = nb[s]; bv = v[s]; }
        bn = __shfl_sync(0xffffffffu, bn, sl);
        if (bn < 0) continue;  // uniform
        const float ux = __shfl_sync(0xffffffffu, bv.x, sl);
        const float uy = __shfl_sync(0xffffffffu, bv.y, sl);
        const float uz = __shfl_sync(0xffffffffu, bv.z, sl);
#pragma unroll
        for (int s = 0; s < S; s++) {
            const int t = lane + 32 * s;
            if (test[s] && keep[s] && jp < t) {
                ++tests;
                const float lx = fs_affine(ax[s], ay[s], az[s], tx[s], ux, uy, uz);
                const float ly = fs_affine(px[s], py[s], pz[s], ty[s], ux, uy, uz);
                const float lz = fs_affine(qx[s], qy[s], qz[s], tz[s], ux, uy, uz);
                // Estimate with a reciprocal (relative error < 1e-6 of the exact
                // expression); the exact divisions decide only near the threshold.
                const float est = __fmaf_rn(lx, lx, __fmul_rn(__fmaf_rn(ly, ly, __fmul_rn(lz, lz)), inv_aa));
                bool inside;
                if (est < dd[s] * 0.99999f) inside = true;
                else if (est > dd[s] * 1.00001f) inside = false;
                else inside = fs_ellipsoid(lx, ly, lz, aa) < dd[s];
                if (inside) keep[s] = false;
            }
        }
    }
    int cnt = 0;
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        if (t < k && nb[s] != -1 && !keep[s]) row[t] = -1;
        cnt += __popc(__ballot_sync(0xffffffffu, keep[s]));
    }
    return cnt;
}

}  // namespace
}  // namespace egt
