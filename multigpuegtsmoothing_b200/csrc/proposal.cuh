// Learned search proposal: definitions shared by the proposal network
// (proposal.cu) and the proposal-driven kNN kernel (knn.cu).
//
// This is an extension of this project; the reference has no counterpart.  A
// proposal class names a box of level-L cells of half-width R around the
// query's level-L cell (classes 0..14, ordered by volume); class 15 means
// "run the plain search".  The box search is accepted only when it provably
// returns the plain search's list (conditions listed in knn.cu).
#pragma once
#include "egt_internal.cuh"
#include "knn_common.cuh"

namespace egt {

constexpr int kPropClasses = 16;
constexpr int kPropPlain = kPropClasses - 1;
constexpr int kPropFeatures = 8;
constexpr int kPropHidden = 32;
// Parameter layout: row-major [out][in] weights, each followed by its bias.
constexpr int kPW1 = 0;
constexpr int kPB1 = kPW1 + kPropHidden * kPropFeatures;
constexpr int kPW2 = kPB1 + kPropHidden;
constexpr int kPB2 = kPW2 + kPropHidden * kPropHidden;
constexpr int kPW3 = kPB2 + kPropHidden;
constexpr int kPB3 = kPW3 + kPropClasses * kPropHidden;
constexpr int kPropParams = kPB3 + kPropClasses;  // 1872
static_assert(kPropParams == EGT_PROPOSAL_PARAMS, "parameter count");

// Margin (normalised units) by which the k-th distance ball must clear every
// in-grid face of a box.  It covers the rounding of the float cell keys
// (< 3e-7) and of the float squared distances.
constexpr double kBoxMargin = 2e-6;
constexpr int kMaxBoxRadius = 6;

// {level, radius} of classes 0..14.
__constant__ static const signed char kBoxClass[kPropPlain][2] = {
    {0, 1}, {0, 2}, {0, 3}, {0, 4}, {0, 5}, {0, 6}, {1, 4}, {1, 5},
    {1, 6}, {2, 4}, {2, 5}, {2, 6}, {3, 4}, {3, 5}, {3, 6}};

// (dy, dz) row offsets of a box, ring by ring (Chebyshev radius, then
// Euclidean): the first (2j+1)^2 entries are exactly the rows of half-width j.
__constant__ static const signed char kRowOrder[(2 * kMaxBoxRadius + 1) * (2 * kMaxBoxRadius + 1)][2] = {
    {0, 0}, {0, -1}, {-1, 0}, {1, 0}, {0, 1}, {-1, -1}, {1, -1}, {-1, 1}, {1, 1}, {0, -2}, {-2, 0}, {2, 0},
    {0, 2}, {-1, -2}, {1, -2}, {-2, -1}, {2, -1}, {-2, 1}, {2, 1}, {-1, 2}, {1, 2}, {-2, -2}, {2, -2}, {-2, 2},
    {2, 2}, {0, -3}, {-3, 0}, {3, 0}, {0, 3}, {-1, -3}, {1, -3}, {-3, -1}, {3, -1}, {-3, 1}, {3, 1}, {-1, 3},
    {1, 3}, {-2, -3}, {2, -3}, {-3, -2}, {3, -2}, {-3, 2}, {3, 2}, {-2, 3}, {2, 3}, {-3, -3}, {3, -3}, {-3, 3},
    {3, 3}, {0, -4}, {-4, 0}, {4, 0}, {0, 4}, {-1, -4}, {1, -4}, {-4, -1}, {4, -1}, {-4, 1}, {4, 1}, {-1, 4},
    {1, 4}, {-2, -4}, {2, -4}, {-4, -2}, {4, -2}, {-4, 2}, {4, 2}, {-2, 4}, {2, 4}, {-3, -4}, {3, -4}, {-4, -3},
    {4, -3}, {-4, 3}, {4, 3}, {-3, 4}, {3, 4}, {-4, -4}, {4, -4}, {-4, 4}, {4, 4}, {0, -5}, {-5, 0}, {5, 0},
    {0, 5}, {-1, -5}, {1, -5}, {-5, -1}, {5, -1}, {-5, 1}, {5, 1}, {-1, 5}, {1, 5}, {-2, -5}, {2, -5}, {-5, -2},
    {5, -2}, {-5, 2}, {5, 2}, {-2, 5}, {2, 5}, {-3, -5}, {3, -5}, {-5, -3}, {5, -3}, {-5, 3}, {5, 3}, {-3, 5},
    {3, 5}, {-4, -5}, {4, -5}, {-5, -4}, {5, -4}, {-5, 4}, {5, 4}, {-4, 5}, {4, 5}, {-5, -5}, {5, -5}, {-5, 5},
    {5, 5}, {0, -6}, {-6, 0}, {6, 0}, {0, 6}, {-1, -6}, {1, -6}, {-6, -1}, {6, -1}, {-6, 1}, {6, 1}, {-1, 6},
    {1, 6}, {-2, -6}, {2, -6}, {-6, -2}, {6, -2}, {-6, 2}, {6, 2}, {-2, 6}, {2, 6}, {-3, -6}, {3, -6}, {-6, -3},
    {6, -3}, {-6, 3}, {6, 3}, {-3, 6}, {3, 6}, {-4, -6}, {4, -6}, {-6, -4}, {6, -4}, {-6, 4}, {6, 4}, {-4, 6},
    {4, 6}, {-5, -6}, {5, -6}, {-6, -5}, {6, -5}, {-6, 5}, {6, 5}, {-5, 6}, {5, 6}, {-6, -6}, {6, -6}, {-6, 6},
    {6, 6}};

// Points of the cells [x0, x1] (clipped to the grid) of row (cy, cz) of a
// level: [start, end) into the level's order; start == end when empty.  The
// cells of a row are contiguous in the level's order (key x + y*B + z*B^2).
__device__ __forceinline__ int2 row_points(const LevelDev& L, int x0, int x1, int cy, int cz) {
    if (cy < 0 || cy >= L.B || cz < 0 || cz >= L.B) return make_int2(0, 0);
    x0 = max(x0, 0);
    x1 = min(x1, L.B - 1);
    if (x0 > x1) return make_int2(0, 0);
    const int2 rr = L.row_range[cy + cz * L.B];
    int lo = rr.x, hi = rr.y;
    while (lo < hi) {  // first cell with x >= x0
        const int mid = (lo + hi) >> 1;
        if (L.cell_x[mid] < x0) lo = mid + 1;
        else hi = mid;
    }
    const int i0 = lo;
    hi = rr.y;
    while (lo < hi) {  // first cell with x > x1
        const int mid = (lo + hi) >> 1;
        if (L.cell_x[mid] <= x1) lo = mid + 1;
        else hi = mid;
    }
    if (lo == i0) return make_int2(0, 0);
    return make_int2(L.cell_start[i0], L.cell_start[lo]);
}

// Level-0 cell range [lo, end) per axis of the box of class `cls` whose
// (y, z) half-width is `ryz` level-L cells (x keeps the class radius).
__device__ __forceinline__ void box_bounds(int cls, int ryz, uint32_t c0, int lo[3], int end[3]) {
    const int L = kBoxClass[cls][0], R = kBoxClass[cls][1];
    const int ci[3] = {(int)(c0 & 1023u) >> L, (int)((c0 >> 10) & 1023u) >> L, (int)((c0 >> 20) & 1023u) >> L};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const int r = d == 0 ? R : ryz;
        lo[d] = (ci[d] - r) * (1 << L);
        end[d] = (ci[d] + r + 1) * (1 << L);
    }
}

// True when the ball of radius sqrt(kth) + margin around the query lies
// inside the box (faces on the grid boundary do not count: no points lie
// beyond them).
__device__ __forceinline__ bool ball_in_box(const NormParams& np, float4 pq, float kth, const int lo[3],
                                            const int end[3]) {
    const double r = sqrt((double)kth) + kBoxMargin;
    const double h0 = (double)__fmul_rn(__fsub_rn(np.b, np.a), 1.0f / 1024.0f);  // exact: power of two
    const double c[3] = {pq.x, pq.y, pq.z};
    bool ok = true;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        if (lo[d] > 0) ok &= r < c[d] - ((double)np.a + lo[d] * h0);
        if (end[d] < 1024) ok &= r < ((double)np.a + end[d] * h0) - c[d];
    }
    return ok;
}

// First step of the plain search (0 = the query's own cell, s >= 1 = the ring
// at level s-1) whose visited block contains level-0 cell pc; 9 = never.
__device__ __forceinline__ int visit_step(uint32_t pc, uint32_t qc) {
    if (pc == qc) return 0;
    const int px = pc & 1023u, py = (pc >> 10) & 1023u, pz = (pc >> 20) & 1023u;
    const int qx = qc & 1023u, qy = (qc >> 10) & 1023u, qz = (qc >> 20) & 1023u;
#pragma unroll
    for (int L = 0; L < kMaxLevels; L++)
        if (abs((px >> L) - (qx >> L)) <= 1 && abs((py >> L) - (qy >> L)) <= 1 && abs((pz >> L) - (qz >> L)) <= 1)
            return L + 1;
    return kMaxLevels + 1;
}

// The 8 proposal features of a query (one thread): log2(1+count)/16 of its own
// cell at levels 0..5 and of its 3x3x3 level-0 block, and twice the smallest
// fractional distance of the query to a face of its level-0 cell.
__device__ __forceinline__ void proposal_features(const LevelDev* lv, const NormParams& np, float4 pq,
                                                  float f[kPropFeatures]) {
    const uint32_t c0 = __float_as_uint(pq.w);
    const int cx = c0 & 1023u, cy = (c0 >> 10) & 1023u, cz = (c0 >> 20) & 1023u;
#pragma unroll
    for (int L = 0; L < 6; L++) {
        const int2 r = find_cell(lv[L], cx >> L, cy >> L, cz >> L);
        const int cnt = r.x >= 0 ? r.y - r.x : 0;
        f[L] = __fmul_rn(log2f(__fadd_rn(1.0f, (float)cnt)), 0.0625f);
    }
    int blk = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; dz++)
#pragma unroll
        for (int dy = -1; dy <= 1; dy++) {
            const int2 r = row_points(lv[0], cx - 1, cx + 1, cy + dy, cz + dz);
            blk += r.y - r.x;
        }
    f[6] = __fmul_rn(log2f(__fadd_rn(1.0f, (float)blk)), 0.0625f);
    const float c[3] = {pq.x, pq.y, pq.z};
    const int ci[3] = {cx, cy, cz};
    float m = 0.5f;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const float v = __fmul_rn(__fdiv_rn(__fsub_rn(c[d], np.a), __fsub_rn(np.b, np.a)), 1024.0f);
        const float fr = __fsub_rn(v, (float)ci[d]);
        m = fminf(m, fminf(fr, __fsub_rn(1.0f, fr)));
    }
    f[7] = __fmul_rn(2.0f, fmaxf(m, 0.0f));
}

// Proposal-network parameters live on the device as binary16 (the weights the
// kernels compute with); FP32 master copies are kept for training.
egt_status proposal_classes(egt_handle* h, const egt_proposal* p);  // fills h->pclass
egt_status level_maxpop(egt_handle* h);                               // fills h->maxpop

}  // namespace egt
