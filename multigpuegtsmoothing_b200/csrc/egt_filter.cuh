// Elliptic-Gabriel filter of one query's list, shared by the single-cloud
// (egt.cu) and batched (batch.cu) kernels.  See egt.cu for the reference
// correspondence.  A query takes a group of G lanes (G = 32: one query per
// warp; G = 16: two, which keeps more lanes busy when k does not fill whole
// 32-slot rounds); slot t of the list sits on lane t % G of the group, round
// t / G.  Every lane of the warp calls it (an `active` false group filters
// nothing and writes nothing).  Returns the number of kept entries (uniform
// over the group); dropped entries of `row` are set to -1.  tests counts the
// ellipsoid tests this lane evaluated; s_v is the group's own staging
// buffer.
#pragma once
#include "egt_internal.cuh"

namespace egt {
namespace {

template <int S, int G = 32>
__device__ __forceinline__ int egt_query(const float4* __restrict__ p4, float4 p, int* __restrict__ row, int k,
                                         float alpha, int lane, unsigned& tests, float4* __restrict__ s_v,
                                         bool active = true) {
    static_assert(G == 16 || G == 32, "groups of 16 or 32 lanes");
    const unsigned gmask = G == 32 ? 0xffffffffu : (0xffffu << (lane & 16));
    lane &= G - 1;  // from here on: the lane within the group
    int nb[S];
    float4 v[S];
    bool keep[S], test[S];
    float ax[S], ay[S], az[S], px[S], py[S], pz[S], qx[S], qy[S], qz[S], tx[S], ty[S], tz[S], dd[S];
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + G * s;
        nb[s] = active && t < k ? row[t] : -1;
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
    // the list's positions, read by the whole warp from shared memory (w: the
    // neighbour index, -1 for an empty slot)
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + G * s;
        if (t < k) s_v[t] = make_float4(v[s].x, v[s].y, v[s].z, __int_as_float(nb[s]));
    }
    __syncwarp();
    // last slot index that still has something to test, over the whole warp
    // (a group past its own last slot tests nothing)
    int hi = -1;
#pragma unroll
    for (int s = 0; s < S; s++)
        if (test[s]) hi = lane + G * s;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    // Is slot s inside the ellipsoid of the closer neighbour u?  Estimated with
    // a reciprocal (relative error < 1e-6 of the exact expression); the exact
    // divisions decide only near the threshold.
    auto inside = [&](int s, float4 u) {
        const float lx = fs_affine(ax[s], ay[s], az[s], tx[s], u.x, u.y, u.z);
        const float ly = fs_affine(px[s], py[s], pz[s], ty[s], u.x, u.y, u.z);
        const float lz = fs_affine(qx[s], qy[s], qz[s], tz[s], u.x, u.y, u.z);
        const float est = __fmaf_rn(lx, lx, __fmul_rn(__fmaf_rn(ly, ly, __fmul_rn(lz, lz)), inv_aa));
        if (est < dd[s] * 0.99999f) return true;
        if (est > dd[s] * 1.00001f) return false;
        return fs_ellipsoid(lx, ly, lz, aa) < dd[s];
    };
    // The closer neighbours in list order, each read once by the whole warp.
    // live[s]: slot s still has tests to run (it is tested and not rejected).
    bool live[S];
#pragma unroll
    for (int s = 0; s < S; s++) live[s] = test[s] && keep[s];
    for (int jp = 0; jp < hi; jp++) {
        if ((jp & 7) == 0) {  // stop once every slot with a pending test is decided
            bool pending = false;
#pragma unroll
            for (int s = 0; s < S; s++) pending |= live[s] && jp < lane + G * s;
            if (!__any_sync(0xffffffffu, pending)) break;
        }
        const float4 u = s_v[jp];  // jp < hi < k
        const bool filled = __float_as_int(u.w) >= 0;  // not an empty slot (uniform over the group)
#pragma unroll
        for (int s = 0; s < S; s++) {
            if (filled && live[s] && jp < lane + G * s) {
                ++tests;
                if (inside(s, u)) { keep[s] = false; live[s] = false; }
            }
        }
    }
    int cnt = 0;
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + G * s;
        if (active && t < k && nb[s] != -1 && !keep[s]) row[t] = -1;
        cnt += __popc(__ballot_sync(0xffffffffu, keep[s]) & gmask);
    }
    return cnt;
}

}  // namespace
}  // namespace egt
