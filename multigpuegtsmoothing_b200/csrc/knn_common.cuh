// Warp-cooperative sorted neighbour list with the reference's insertion rule.
//
// The list of a query is held in registers across the 32 lanes of a warp:
// slot t lives in lane t % 32, register t / 32 (S registers per lane, k <= 32*S).
// insert() reproduces newNeighborSearch::appendDistanceGrid
// (GridKNNCuda.cu:311-339) exactly:
//   * admit only if d < list[k-1] (the list is pre-filled with 1e10, so this is
//     "always" while the list is not full, and strict at the k-th slot);
//   * reject an index already among the first `counter` slots;
//   * insert at FindPosition(list, d, 0, counter-1) (GridKNNCuda.cu:126-143): the
//     binary search returns the slot of the first equal element it meets, or
//     the insertion point -- equal distances therefore land where that search
//     lands, not simply after the existing ones;
//   * shift the tail down by one, dropping slot k-1 when the list is full.
// All lanes call insert() with the same (d, p): control flow stays uniform.
#pragma once
#include "egt_internal.cuh"

namespace egt {

template <int S>
struct WarpList {
    float dist[S];
    int idx[S];
    int counter;  // number of filled slots (uniform)
    float kth;    // value of slot k-1 (uniform): 1e10 until the list is full
    int k;
    bool tie;     // an insertion met an equal distance already in the list
    unsigned ev = 0;  // candidate distances this lane evaluated (not reset by init)

    __device__ __forceinline__ void init(int k_) {
#pragma unroll
        for (int s = 0; s < S; s++) { dist[s] = 1e10f; idx[s] = -1; }
        counter = 0;
        kth = 1e10f;
        k = k_;
        tie = false;
    }

    __device__ __forceinline__ float fetch_dist(int t) const {
        float v = dist[0];
#pragma unroll
        for (int s = 1; s < S; s++)
            if ((t >> 5) == s) v = dist[s];
        return __shfl_sync(0xffffffffu, v, t & 31);
    }

    __device__ __forceinline__ void insert(float d, int p, int lane) {
        if (!(d < kth)) return;
        // dedup among the filled slots
        bool dup = false, eq = false;
        unsigned lt = 0;
#pragma unroll
        for (int s = 0; s < S; s++) {
            const int t = lane + 32 * s;
            const bool live = t < counter;
            dup |= live && idx[s] == p;
            eq |= live && dist[s] == d;
            lt += __popc(__ballot_sync(0xffffffffu, live && dist[s] < d));
        }
        if (__any_sync(0xffffffffu, dup)) return;
        int pos;
        if (!__any_sync(0xffffffffu, eq)) {
            pos = (int)lt;  // no equal element: FindPosition returns the insertion point
        } else {
            tie = true;
            int low = 0, high = counter - 1;
            pos = -1;
            while (low <= high) {  // at most log2(k)+1 iterations
                const int mid = low + (high - low) / 2;
                const float a = fetch_dist(mid);
                if (a == d) { pos = mid; break; }
                if (a < d) low = mid + 1;
                else high = mid - 1;
            }
            if (pos < 0) pos = low + (high - low) / 2;
        }
        // previous slot values (t-1) for the shift, taken before any update
        float pd[S];
        int pi[S];
#pragma unroll
        for (int s = 0; s < S; s++) {
            float up_d = __shfl_up_sync(0xffffffffu, dist[s], 1);
            int up_i = __shfl_up_sync(0xffffffffu, idx[s], 1);
            float wrap_d = __shfl_sync(0xffffffffu, s > 0 ? dist[s > 0 ? s - 1 : 0] : 0.f, 31);
            int wrap_i = __shfl_sync(0xffffffffu, s > 0 ? idx[s > 0 ? s - 1 : 0] : 0, 31);
            pd[s] = lane == 0 ? wrap_d : up_d;
            pi[s] = lane == 0 ? wrap_i : up_i;
        }
#pragma unroll
        for (int s = 0; s < S; s++) {
            const int t = lane + 32 * s;
            if (t < k) {
                if (t == pos) { dist[s] = d; idx[s] = p; }
                else if (t > pos) { dist[s] = pd[s]; idx[s] = pi[s]; }
            }
        }
        counter = counter == k ? k : counter + 1;
        kth = fetch_dist(k - 1);
    }
};

// Sorted insertion without the reference's dedup and tie rules, for candidate
// streams that offer each point once and whose results are discarded when
// two kept distances are equal: admit if d < list[k-1], insert after the
// elements smaller than d.
template <int S>
__device__ __forceinline__ void insert_sorted(WarpList<S>& L, float d, int p, int lane) {
    if (!(d < L.kth)) return;
    unsigned lt = 0;
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        lt += __popc(__ballot_sync(0xffffffffu, t < L.counter && L.dist[s] < d));
    }
    const int pos = (int)lt;
    float pd[S];
    int pi[S];
#pragma unroll
    for (int s = 0; s < S; s++) {
        float up_d = __shfl_up_sync(0xffffffffu, L.dist[s], 1);
        int up_i = __shfl_up_sync(0xffffffffu, L.idx[s], 1);
        float wrap_d = __shfl_sync(0xffffffffu, s > 0 ? L.dist[s > 0 ? s - 1 : 0] : 0.f, 31);
        int wrap_i = __shfl_sync(0xffffffffu, s > 0 ? L.idx[s > 0 ? s - 1 : 0] : 0, 31);
        pd[s] = lane == 0 ? wrap_d : up_d;
        pi[s] = lane == 0 ? wrap_i : up_i;
    }
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        if (t < L.k) {
            if (t == pos) { L.dist[s] = d; L.idx[s] = p; }
            else if (t > pos) { L.dist[s] = pd[s]; L.idx[s] = pi[s]; }
        }
    }
    L.counter = L.counter == L.k ? L.k : L.counter + 1;
    L.kth = L.fetch_dist(L.k - 1);
}

// Warp bitonic sort of one (d, p) pair per lane, ascending in d across lanes.
__device__ __forceinline__ void warp_sort32(float& d, int& p, int lane) {
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const float od = __shfl_xor_sync(0xffffffffu, d, stride);
            const int op = __shfl_xor_sync(0xffffffffu, p, stride);
            const bool keep_min = ((lane & stride) == 0) == ((lane & size) == 0);
            if (keep_min ? (od < d) : (od > d)) { d = od; p = op; }
        }
    }
}

// Value of slot m of the list, m chosen per lane.
template <int S>
__device__ __forceinline__ float list_dist_at(const WarpList<S>& L, int m) {
    float v = 0.0f;
#pragma unroll
    for (int s = 0; s < S; s++) {
        const float u = __shfl_sync(0xffffffffu, L.dist[s], m & 31);
        if ((m >> 5) == s) v = u;
    }
    return v;
}

// Merges the lanes' admitted candidates (ok) into the sorted list in one
// step: the batch is sorted by a warp bitonic network, every element's slot
// in the merged order is found by binary search in the other sequence, and
// the merged prefix is exchanged through shared memory (sd/sp: 32*S slots
// owned by the calling warp).  Equal distances place the list's element
// first.  The result is the sorted L.k smallest of list + batch, like L.k
// insert_sorted calls, so it serves the same (tie-free) candidate streams.
template <int S>
__device__ __forceinline__ void merge_batch(WarpList<S>& L, float d, int p, bool ok, int lane, float* sd, int* sp) {
    float bd = ok ? d : 3.0e38f;
    int bp = p;
    const int nb = __popc(__ballot_sync(0xffffffffu, ok));
    warp_sort32(bd, bp, lane);
    const int cnt = L.counter, cap = L.k;
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        const float x = L.dist[s];
        int lo = 0, hi = nb;  // batch elements < x
#pragma unroll
        for (int it = 0; it < 6; it++) {
            const int mid = (lo + hi) >> 1;
            const float v = __shfl_sync(0xffffffffu, bd, mid & 31);
            if (lo < hi) {
                if (v < x) lo = mid + 1;
                else hi = mid;
            }
        }
        const int r = t + lo;
        if (t < cnt && r < cap) { sd[r] = x; sp[r] = L.idx[s]; }
    }
    {
        int lo = 0, hi = cnt;  // list elements <= bd
#pragma unroll
        for (int it = 0; it < 9; it++) {  // cnt <= 256
            const int mid = (lo + hi) >> 1;
            const float v = list_dist_at(L, mid);
            if (lo < hi) {
                if (v <= bd) lo = mid + 1;
                else hi = mid;
            }
        }
        const int r = lane + lo;
        if (lane < nb && r < cap) { sd[r] = bd; sp[r] = bp; }
    }
    __syncwarp();
    const int nc = min(cnt + nb, cap);
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        if (t < nc) { L.dist[s] = sd[t]; L.idx[s] = sp[t]; }
    }
    __syncwarp();
    L.counter = nc;
    L.kth = L.fetch_dist(cap - 1);
}

// Merges a small batch of admitted candidates (ok; `mask` = their lanes)
// into the sorted list without sorting the batch: each candidate's slot is
// the number of list elements <= its distance (one binary search per lane)
// plus the number of candidates ordered before it (distance, then lane); each
// list element moves down by the number of candidates below it.  Equal
// distances place the list's element first and candidates in lane order, as
// merge_batch does up to the order of equal batch elements, which only the
// tie-free candidate streams of merge_batch reach.  Cost: one binary search
// plus a few instructions per candidate, against a full 32-wide sort.
template <int S>
__device__ __forceinline__ void merge_rank(WarpList<S>& L, float d, int p, bool ok, unsigned mask, int lane,
                                           float* sd, int* sp) {
    constexpr int kSteps = S <= 1 ? 6 : S <= 2 ? 7 : S <= 4 ? 8 : 9;  // > log2(32*S)
    const int cnt = L.counter, cap = L.k;
    int lo = 0, hi = cnt;  // list elements <= d
#pragma unroll
    for (int it = 0; it < kSteps; it++) {
        const int mid = (lo + hi) >> 1;
        const float v = list_dist_at(L, mid);
        if (lo < hi) {
            if (v <= d) lo = mid + 1;
            else hi = mid;
        }
    }
    int rank = lo;
    int sh[S];
#pragma unroll
    for (int s = 0; s < S; s++) sh[s] = 0;
    for (unsigned m = mask; m; m &= m - 1) {
        const int src = __ffs(m) - 1;
        const float dj = __shfl_sync(0xffffffffu, d, src);
        rank += (dj < d || (dj == d && src < lane)) ? 1 : 0;
#pragma unroll
        for (int s = 0; s < S; s++) sh[s] += dj < L.dist[s] ? 1 : 0;
    }
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s, r = t + sh[s];
        if (t < cnt && r < cap) { sd[r] = L.dist[s]; sp[r] = L.idx[s]; }
    }
    if (ok && rank < cap) { sd[rank] = d; sp[rank] = p; }
    __syncwarp();
    const int nc = min(cnt + __popc(mask), cap);
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        if (t < nc) { L.dist[s] = sd[t]; L.idx[s] = sp[t]; }
    }
    __syncwarp();
    L.counter = nc;
    L.kth = L.fetch_dist(cap - 1);
}

// Locate cell (cx,cy,cz) of a level: returns [start,end) into the level's
// order array, or start == end == -1 when the cell is empty / out of range.
__device__ __forceinline__ int2 find_cell(const LevelDev& L, int cx, int cy, int cz) {
    const int B = L.B;
    if (cx < 0 || cx >= B || cy < 0 || cy >= B || cz < 0 || cz >= B) return make_int2(-1, -1);
    const int2 rr = L.row_range[cy + cz * B];
    int lo = rr.x, hi = rr.y;
    while (lo < hi) {  // at most log2(B)+1 iterations
        const int mid = (lo + hi) >> 1;
        if (L.cell_x[mid] < cx) lo = mid + 1;
        else hi = mid;
    }
    if (lo < rr.y && L.cell_x[lo] == cx) return make_int2(L.cell_start[lo], L.cell_start[lo + 1]);
    return make_int2(-1, -1);
}

// Shell order of GRIDCUDAKNNSELF_COMPACT for offset 1 (GridKNNCuda.cu:2480-2551).
__constant__ static const signed char kShell[26][3] = {
    {0, 0, -1}, {0, 0, 1},
    {0, -1, 0}, {0, 1, 0},
    {-1, 0, 0}, {1, 0, 0},
    {-1, -1, 0}, {-1, 1, 0}, {1, -1, 0}, {1, 1, 0},
    {-1, 0, -1}, {-1, 0, 1}, {1, 0, -1}, {1, 0, 1},
    {0, -1, -1}, {0, -1, 1}, {0, 1, -1}, {0, 1, 1},
    {-1, -1, -1}, {-1, -1, 1}, {-1, 1, -1}, {-1, 1, 1}, {1, -1, -1}, {1, -1, 1}, {1, 1, -1}, {1, 1, 1},
};

}  // namespace egt
