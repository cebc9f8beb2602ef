// Exact self-kNN over the cell hierarchy with the reference's semantics.
//
// Reference: GridStructure::GRIDCUDAKNNSELF_COMPACT (GridKNNCuda.cu:2322-2634)
// and its kernel construct_neighbors_self_compact (GridKNNCuda.cu:647-743).
// The reference runs one launch per shell cell (27 launches for the own cell
// and ring 1, 26 per further level), each followed by a device sync, a host
// reduction and a compaction of the still-searching queries.  Here one warp
// runs a query through the whole sequence in a single launch:
//
//   own level-0 cell; decide; ring 1 at level 0; decide; ring 1 at level 1; ...
//   ring 1 at level 7 (B = 8); a query still searching after that is invalid.
//
// The candidate order is the reference's: cells in its shell nest order, the
// points of a cell in ascending sorted index (the stable level sort), and the
// list is updated by the exact appendDistanceGrid rule (knn_common.cuh), so
// the produced lists -- including the order of equal distances -- are
// bit-identical to the reference's.  The 26 shell cells of a level are
// resolved in parallel (one per lane) and their points are streamed as one
// flattened candidate sequence, 32 candidates per step.
//
// Re-visits are skipped: the cells visited up to level L-1 form the 3x3x3
// block of level L-1 around the query, and the level-L ring covers it again.
// A point of that block was already offered to the list: it is either in the
// list (the dedup rule rejects it) or farther than the k-th distance of that
// time, which never grows (the admission rule rejects it), so offering it again
// cannot change the list.
#include "egt_internal.cuh"
#include "knn_common.cuh"

namespace egt {
namespace {

struct KnnArgs {
    const float4* __restrict__ p4;
    const NormParams* __restrict__ np;
    LevelDev lv[kMaxLevels];
    int n, k, max_pts;
    int* __restrict__ lists;
    float* __restrict__ kth_out;
    uint8_t* __restrict__ qlevel;
    unsigned long long* __restrict__ counters;
};

constexpr int kWarps = 8;

// Continue decision after the last cube of a shell (GridKNNCuda.cu:694-741).
__device__ __forceinline__ bool decide(const NormParams& np, int L, int o, int counter, int k, float kth,
                                       bool invalid, float4 q, int cx0, int cy0, int cz0) {
    if (invalid) return false;
    const int B = 1024 >> L;
    const float h = __fdiv_rn(__fsub_rn(np.b, np.a), (float)B);
    const float c[3] = {q.x, q.y, q.z};
    const int ci[3] = {cx0 >> L, cy0 >> L, cz0 >> L};
    if (counter < k) {
        const float st = __fsqrt_rn(np.thres);
        bool more = false;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            more |= (ci[d] - o >= 0) && st > fs_face_lo(c[d], np.a, (float)(ci[d] - o), h);
            more |= (ci[d] + o + 1 <= B) && st > fs_face_hi(c[d], np.a, (float)(ci[d] + o + 1), h);
        }
        return more;
    }
    const float r = __fsqrt_rn(kth);
    bool more = false;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        more |= (ci[d] - o >= 0) && r >= fs_face_lo(c[d], np.a, (float)(ci[d] - o), h);
        more |= (ci[d] + o + 1 <= B) && r >= fs_face_hi(c[d], np.a, (float)(ci[d] + o + 1), h);
    }
    return more;
}

// Streams the points of `m` cells (cell l held by lane l as [cs, ce), ce < 0 =
// empty) through the list, in cell order.  Sets `invalid` when a visited cell
// holds >= max_pts points (GridKNNCuda.cu:672, 685): the cells before it are
// still processed, the rest are not.  skipL >= 0: skip points whose level-skipL
// cell lies in the 3x3x3 block around the query's (already visited).
template <int S>
__device__ __forceinline__ void stream_cells(WarpList<S>& L, bool& invalid, int m, int cs, int ce,
                                             const int* __restrict__ order, const float4* __restrict__ p4,
                                             int q, float4 pq, float thres, int max_pts, int lane,
                                             int skipL, uint32_t qc0, int* s_pref, int* s_start) {
    const bool exists = lane < m && ce >= 0;
    const bool big = exists && (ce - cs) >= max_pts;
    const unsigned bigmask = __ballot_sync(0xffffffffu, big);
    const int mlim = bigmask ? (__ffs(bigmask) - 1) : m;
    int sz = (lane < mlim && exists) ? ce - cs : 0;
    int incl = sz;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    __syncwarp();
    s_pref[lane] = incl;
    s_start[lane] = cs;
    __syncwarp();
    const int qx = (int)((qc0 & 1023u) >> max(skipL, 0)), qy = (int)(((qc0 >> 10) & 1023u) >> max(skipL, 0)),
              qz = (int)(((qc0 >> 20) & 1023u) >> max(skipL, 0));
    for (int base = 0; base < total; base += 32) {
        const int j = base + lane;
        float d = 1e30f;
        int p = -1;
        bool ok = false;
        if (j < total) {
            int lo = 0, hi = mlim - 1;  // first cell with incl > j
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (s_pref[mid] > j) hi = mid;
                else lo = mid + 1;
            }
            const int excl = lo > 0 ? s_pref[lo - 1] : 0;
            const int pos = s_start[lo] + (j - excl);
            p = order ? order[pos] : pos;
            if (p != q) {
                const float4 v = p4[p];
                bool fresh = true;
                if (skipL >= 0) {
                    const uint32_t c = __float_as_uint(v.w);
                    const int px = (int)((c & 1023u) >> skipL), py = (int)(((c >> 10) & 1023u) >> skipL),
                              pz = (int)(((c >> 20) & 1023u) >> skipL);
                    fresh = abs(px - qx) > 1 || abs(py - qy) > 1 || abs(pz - qz) > 1;
                }
                if (fresh) {
                    d = fs_dist3(pq.x, pq.y, pq.z, v.x, v.y, v.z);
                    ok = d <= thres;
                }
            }
        }
        unsigned mask = __ballot_sync(0xffffffffu, ok && d < L.kth);
        while (mask) {
            const int src = __ffs(mask) - 1;
            mask &= mask - 1;
            const float dd = __shfl_sync(0xffffffffu, d, src);
            const int pp = __shfl_sync(0xffffffffu, p, src);
            L.insert(dd, pp, lane);
        }
    }
    if (bigmask) invalid = true;
}

// The whole reference search for query q.  Returns the level reached
// (kMaxLevels when the query ran out of levels).
template <int S>
__device__ int search(const KnnArgs& a, const NormParams& np, int q, float4 pq, WarpList<S>& L,
                      bool& invalid, int lane, int* s_pref, int* s_start) {
    const uint32_t c0 = __float_as_uint(pq.w);
    const int cx0 = c0 & 1023, cy0 = (c0 >> 10) & 1023, cz0 = (c0 >> 20) & 1023;
    L.init(a.k);
    invalid = false;
    // offset 0 at level 0: the query's own cell (always occupied)
    int2 own = lane == 0 ? find_cell(a.lv[0], cx0, cy0, cz0) : make_int2(-1, -1);
    stream_cells<S>(L, invalid, 1, own.x, own.y, nullptr, a.p4, q, pq, np.thres, a.max_pts, lane, -1, c0, s_pref,
                    s_start);
    bool cont = decide(np, 0, 0, L.counter, L.k, L.kth, invalid, pq, cx0, cy0, cz0);
    int reached = 0;
    for (int lvl = 0; cont; lvl++) {
        reached = lvl;
        const LevelDev& LV = a.lv[lvl];
        int2 cell = make_int2(-1, -1);
        if (lane < 26)
            cell = find_cell(LV, (cx0 >> lvl) + kShell[lane][0], (cy0 >> lvl) + kShell[lane][1],
                             (cz0 >> lvl) + kShell[lane][2]);
        stream_cells<S>(L, invalid, 26, cell.x, cell.y, LV.order, a.p4, q, pq, np.thres, a.max_pts, lane, lvl - 1,
                        c0, s_pref, s_start);
        cont = decide(np, lvl, 1, L.counter, L.k, L.kth, invalid, pq, cx0, cy0, cz0);
        if (lvl == kMaxLevels - 1) break;
    }
    // still searching after the B = 8 ring: invalid (GridKNNCuda.cu:2572-2586)
    if (cont) { invalid = true; reached = kMaxLevels; }
    return reached;
}

template <int S>
__global__ void __launch_bounds__(kWarps * 32) k_knn_plain(KnnArgs a) {
    __shared__ int s_pref[kWarps][32];
    __shared__ int s_start[kWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int q = blockIdx.x * kWarps + w;
    if (q >= a.n) return;
    const NormParams np = *a.np;
    const float4 pq = a.p4[q];
    WarpList<S> L;
    bool invalid;
    const int reached = search<S>(a, np, q, pq, L, invalid, lane, s_pref[w], s_start[w]);
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        if (t < a.k) a.lists[(size_t)q * a.k + t] = invalid ? -1 : L.idx[s];
    }
    if (lane == 0) {
        if (a.kth_out) a.kth_out[q] = (!invalid && L.counter == a.k) ? L.kth : 1e10f;
        if (a.qlevel) a.qlevel[q] = (uint8_t)reached;
        if (invalid) atomicAdd(&a.counters[kCtrInvalid], 1ull);
        atomicMax(&a.counters[kCtrMaxLevel], (unsigned long long)reached);
    }
}

template <int S>
egt_status launch(const KnnArgs& a, cudaStream_t st) {
    const unsigned G = (unsigned)((a.n + kWarps - 1) / kWarps);
    k_knn_plain<S><<<G, kWarps * 32, 0, st>>>(a);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

}  // namespace

egt_status run_knn(egt_handle* h, int k) {
    if (k <= 0 || k > 256) { set_error("egt_knn: k must be in [1, 256]"); return EGT_ERR_ARG; }
    if (h->levels_built < kMaxLevels) { set_error("egt_knn: grid hierarchy not built"); return EGT_ERR_STATE; }
    cudaStream_t st = h->stream;
    const int64_t n = h->n;
    if (h->k != k || !h->lists) {
        if (h->lists) dev_free(h, h->lists);
        h->lists = nullptr;
        EGT_CUDA_TRY(dev_alloc(h, &h->lists, sizeof(int) * (size_t)n * k));
        h->k = k;
    }
    if (!h->kth) EGT_CUDA_TRY(dev_alloc(h, &h->kth, sizeof(float) * n));
    if (!h->qlevel) EGT_CUDA_TRY(dev_alloc(h, &h->qlevel, n));
    h->have_csr = false;
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrInvalid, 0, 2 * sizeof(unsigned long long), st));
    KnnArgs a;
    a.p4 = h->p4;
    a.np = h->d_norm;
    for (int L = 0; L < kMaxLevels; L++) a.lv[L] = h->lv[L];
    a.n = (int)n;
    a.k = k;
    a.max_pts = h->cfg.max_points_in_cell;
    a.lists = h->lists;
    a.kth_out = h->kth;
    a.qlevel = h->qlevel;
    a.counters = h->d_counters;
    EGT_CUDA_TRY(cudaEventRecord(h->ev[2], st));
    if (k <= 32) EGT_TRY(launch<1>(a, st));
    else if (k <= 64) EGT_TRY(launch<2>(a, st));
    else if (k <= 128) EGT_TRY(launch<4>(a, st));
    else EGT_TRY(launch<8>(a, st));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[3], st));
    return EGT_OK;
}

}  // namespace egt
