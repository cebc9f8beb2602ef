// Normal orientation over a minimum spanning forest.
//
// Reference: Normal_CUDA::GetNormals (Normal_CUDA.cu:329-711) with CUDA_MST.cu
// (Borůvka, :296-418) and bfs.cu (level-synchronous BFS with a host loop per
// level, :63-110).  The reference builds undirected edges (min,max) from the
// filtered lists with weight max(0, 1 - |n_u . n_v|), removes duplicates by the
// key u*n+v, sorts by weight (stable, so ties stay in key order), takes a
// minimum spanning forest and walks each tree breadth-first from a root,
// negating a child's normal when its dot product with its parent's (already
// oriented) normal is negative.  The first root is the first vertex of the
// lightest edge (Normal_CUDA.cu:438-440).
//
// Along a tree path the BFS rule makes the sign of every vertex a product of
// the edge signs sign(n_u . n_v) from the root, so no traversal order is
// needed: this file runs a deterministic Borůvka that carries that sign parity
// through its component merges (each vertex stores its sign relative to its
// component representative, merged by pointer jumping), then re-bases every
// tree on its root.  Edges are totally ordered by (weight, key) -- the
// reference's sort order -- so the forest is the unique minimum one for that
// order.  Every tree is rooted at the first vertex of its lightest edge (for
// the first tree this is the reference's root; the reference picks later roots
// by a racy last-writer search, Normal_CUDA.cu:232-240).  An exactly zero dot
// product is treated as a same-sign link (the reference re-seeds the child from
// its raw sign there).  Component sign votes (Normal_CUDA.cu:517-711) only act
// on list edges that join different trees; the trees are the connected
// components of the list graph, so there are none to act on.
#include <cub/cub.cuh>
#include <numeric>
#include <vector>
#include "egt_internal.cuh"

namespace egt {
namespace {

constexpr unsigned long long kNone = ~0ull;

// Warp-aggregated counter increment: one atomic per warp.  Every lane of the
// warp must call it (pred false for lanes without an item).
__device__ __forceinline__ void warp_count(unsigned long long* ctr, bool pred) {
    const unsigned b = __ballot_sync(0xffffffffu, pred);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(ctr, (unsigned long long)__popc(b));
}

__global__ void k_edge_keys(const int* __restrict__ off, const int* __restrict__ col, int n, int bits,
                            unsigned long long* __restrict__ key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long sentinel = (1ull << (2 * bits)) - 1ull;
    for (int e = off[i]; e < off[i + 1]; e++) {
        const int m = col[e];
        const unsigned u = (unsigned)min(i, m), v = (unsigned)max(i, m);
        key[e] = (u == v) ? sentinel : (((unsigned long long)u << bits) | v);
    }
}

// 1 for the first copy of each edge key in the sorted array (self-loop
// sentinels excluded).
__global__ void k_first_copy(const unsigned long long* __restrict__ key, int64_t m, int bits,
                             unsigned char* __restrict__ flag) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const unsigned long long k = key[e];
    flag[e] = (k != (1ull << (2 * bits)) - 1ull) && (e == 0 || key[e - 1] != k);
}

// Edge e's order key (weight bits, e) -- e is the rank of the edge's vertex
// key, so this is the reference's (weight, key) order -- and its sign.
__global__ void k_edge_init(const unsigned long long* __restrict__ ukey, int E, int bits,
                            const float* __restrict__ nrm, int n, unsigned long long* __restrict__ ckey,
                            signed char* __restrict__ sgn) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const unsigned long long k = ukey[e];
    const int u = (int)(k >> bits), v = (int)(k & ((1ull << bits) - 1ull));
    const float d = fs_dot3(nrm[u], nrm[n + u], nrm[2 * (size_t)n + u], nrm[v], nrm[n + v], nrm[2 * (size_t)n + v]);
    const float w = fmaxf(0.0f, __fsub_rn(1.0f, fabsf(d)));
    ckey[e] = ((unsigned long long)__float_as_uint(w) << 32) | (unsigned)e;
    sgn[e] = d < 0.0f ? -1 : 1;
}

__global__ void k_init_comp(int n, int* __restrict__ comp, signed char* __restrict__ sig) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    comp[v] = v;
    sig[v] = 1;
}

// Lightest live edge of every component.  act: order keys of the edges that
// joined two components at the start of the round (*live of them).
__global__ void k_select(const unsigned long long* __restrict__ act, const int* __restrict__ live,
                         const unsigned long long* __restrict__ ukey, int bits, const int* __restrict__ comp,
                         unsigned long long* __restrict__ best) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *live) return;
    const unsigned long long c = act[i];
    const unsigned long long k = ukey[c & 0xffffffffull];
    const int u = (int)(k >> bits), v = (int)(k & ((1ull << bits) - 1ull));
    const int cu = comp[u], cv = comp[v];
    if (cu == cv) return;
    atomicMin(&best[cu], c);
    atomicMin(&best[cv], c);
}

// Hooks every component to the one across its lightest edge.  A pair that
// chose each other links only the larger representative.  Counts the links
// (= forest edges added) into ctr[kCtrFlag] and ctr[kCtrMsf].
__global__ void k_hook(const unsigned long long* __restrict__ ukey, const signed char* __restrict__ sgn, int n,
                       int bits, const int* __restrict__ comp, const signed char* __restrict__ sig,
                       const unsigned long long* __restrict__ best, int* __restrict__ link,
                       signed char* __restrict__ lpar, unsigned long long* __restrict__ ctr,
                       unsigned char* __restrict__ msf) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    bool linked = false;
    if (c < n) {
        link[c] = c;
        lpar[c] = 1;
        const unsigned long long b = comp[c] == c ? best[c] : kNone;
        if (b != kNone) {
            const int e = (int)(b & 0xffffffffull);
            const unsigned long long k = ukey[e];
            const int u = (int)(k >> bits), v = (int)(k & ((1ull << bits) - 1ull));
            const int x = comp[u] == c ? u : v;
            const int y = x == u ? v : u;
            const int c2 = comp[y];
            if (!(best[c2] == b && c < c2)) {  // mutual choice: the smaller representative stays a root
                link[c] = c2;
                lpar[c] = (signed char)(sig[x] * sgn[e] * sig[y]);
                linked = true;
                if (msf) msf[e] = 1;
            }
        }
    }
    warp_count(&ctr[kCtrFlag], linked);
    warp_count(&ctr[kCtrMsf], linked);
}

__global__ void k_jump(const int* __restrict__ link, const signed char* __restrict__ lpar, int n,
                       int* __restrict__ link2, signed char* __restrict__ lpar2, unsigned long long* __restrict__ ctr) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    bool moved = false;
    if (c < n) {
        const int l = link[c];
        const int ll = link[l];
        moved = l != ll;
        link2[c] = ll;
        lpar2[c] = moved ? (signed char)(lpar[c] * lpar[l]) : lpar[c];
    }
    warp_count(&ctr[kCtrFlag], moved);
}

__global__ void k_relabel(int n, const int* __restrict__ link, const signed char* __restrict__ lpar,
                          int* __restrict__ comp, signed char* __restrict__ sig) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int c = comp[v];
    comp[v] = link[c];
    sig[v] = (signed char)(sig[v] * lpar[c]);
}

// An edge that still joins two components.
struct JoinsTwo {
    const unsigned long long* ukey;
    const int* comp;
    int bits;
    __device__ bool operator()(unsigned long long c) const {
        const unsigned long long k = ukey[c & 0xffffffffull];
        return comp[(int)(k >> bits)] != comp[(int)(k & ((1ull << bits) - 1ull))];
    }
};

// Lightest edge of every tree.  It is the lightest edge at one of its ends, so
// it is the minimum of the first round's choices (first) over the tree's
// vertices.  Lanes of a warp that share a tree combine before the atomic.
__global__ void k_roots(int n, const int* __restrict__ comp, const unsigned long long* __restrict__ first,
                        unsigned long long* __restrict__ rootkey) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = v < n ? comp[v] : -1;
    unsigned long long b = v < n ? first[v] : kNone;
    if (__match_any_sync(0xffffffffu, c) == 0xffffffffu) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long t = __shfl_xor_sync(0xffffffffu, b, o);
            b = t < b ? t : b;
        }
        if ((threadIdx.x & 31) == 0 && c >= 0 && b != kNone) atomicMin(&rootkey[c], b);
    } else if (c >= 0 && b != kNone) {
        atomicMin(&rootkey[c], b);
    }
}

__global__ void k_apply(int n, int bits, const int* __restrict__ comp, const signed char* __restrict__ sig,
                        const unsigned long long* __restrict__ rootkey, const unsigned long long* __restrict__ ukey,
                        float* __restrict__ nrm, unsigned long long* __restrict__ ctr) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    bool root = false;
    if (v < n) {
        const int c = comp[v];
        const unsigned long long rk = rootkey[c];
        if (rk != kNone) {  // else: no edge, keeps its unoriented normal
            const int e = (int)(rk & 0xffffffffull);
            const int R = (int)(ukey[e] >> bits);
            root = v == c;
            if (sig[v] * sig[R] < 0) {
                nrm[v] = -nrm[v];
                nrm[n + v] = -nrm[n + v];
                nrm[2 * (size_t)n + v] = -nrm[2 * (size_t)n + v];
            }
        }
    }
    warp_count(&ctr[kCtrComps], root);
}

// ---- orient_kruskal (MST.cpp:399-423): the reference's CPU orienter ----

// Vertex keys (min << bits | max) of the first k_use entries of every row
// (rows of k ints); empty entries (< 0) and self pairs get the sentinel
// that sorts last.  An entry >= n sets ctr[kCtrFlag].
__global__ void k_kr_keys(const int* __restrict__ knn, int n, int k, int k_use, int bits,
                          unsigned long long* __restrict__ key, unsigned long long* __restrict__ ctr) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * k_use) return;
    const int i = (int)(t / k_use);
    const int m = knn[(int64_t)i * k + (int)(t - (int64_t)i * k_use)];
    const unsigned long long sentinel = (1ull << (2 * bits)) - 1ull;
    if (m >= n) {
        ctr[kCtrFlag] = 1;
        key[t] = sentinel;
        return;
    }
    if (m < 0 || m == i) { key[t] = sentinel; return; }
    const unsigned u = (unsigned)min(i, m), v = (unsigned)max(i, m);
    key[t] = ((unsigned long long)u << bits) | v;
}

// Edge weight max(0, 1 - |d|) in double, d the float dot product
// nx_u*nx_v + ny_u*ny_v + nz_u*nz_v summed left to right with every product
// and sum rounded separately (the reference's host arithmetic, MST.cpp:408-409);
// the weight's bit pattern orders like the weight (it is never negative).
// sgn = -1 for d < 0; zero = 1 for d == 0.
__global__ void k_kr_weights(const unsigned long long* __restrict__ ukey, int E, int bits, const float* __restrict__ nrm,
                             int n, unsigned long long* __restrict__ wkey, int* __restrict__ eidx,
                             signed char* __restrict__ sgn, unsigned char* __restrict__ zero) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const unsigned long long k = ukey[e];
    const int u = (int)(k >> bits), v = (int)(k & ((1ull << bits) - 1ull));
    const float* X = nrm;
    const float* Y = nrm + n;
    const float* Z = nrm + 2 * (size_t)n;
    const float d = __fadd_rn(__fadd_rn(__fmul_rn(X[u], X[v]), __fmul_rn(Y[u], Y[v])), __fmul_rn(Z[u], Z[v]));
    const double w1 = __dsub_rn(1.0, fabs((double)d));
    const double w = w1 > 0.0 ? w1 : 0.0;  // std::max(0.0, w1): +0 for -0 and NaN
    wkey[e] = (unsigned long long)__double_as_longlong(w);
    eidx[e] = e;
    sgn[e] = d < 0.0f ? -1 : 1;
    zero[e] = d == 0.0f;
}

// Order keys (rank << 32 | edge) from the edges sorted by (weight, u, v).
__global__ void k_kr_rank(const int* __restrict__ order, int E, unsigned long long* __restrict__ act) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= E) return;
    act[r] = ((unsigned long long)r << 32) | (unsigned)order[r];
}

// Per rank: the edge's vertex key, and flags for forest edges (f1), forest
// edges with a non-zero dot product (f2, with their order keys in okey) and
// forest edges with a zero dot product (f3).
__global__ void k_kr_forest_lists(const int* __restrict__ order, int E, const unsigned long long* __restrict__ ukey,
                                  const unsigned char* __restrict__ msf, const unsigned char* __restrict__ zero,
                                  unsigned long long* __restrict__ vkey, unsigned long long* __restrict__ okey,
                                  unsigned char* __restrict__ f1, unsigned char* __restrict__ f2,
                                  unsigned char* __restrict__ f3) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= E) return;
    const int e = order[r];
    vkey[r] = ukey[e];
    okey[r] = ((unsigned long long)r << 32) | (unsigned)e;
    const bool in = msf[e] != 0;
    f1[r] = in;
    f2[r] = in && !zero[e];
    f3[r] = in && zero[e];
}

// ref[comp[s]] = s for every walk start s (one per component of comp).
__global__ void k_kr_starts(const int* __restrict__ starts, int ns, const int* __restrict__ comp,
                            int* __restrict__ ref) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    const int s = starts[i];
    ref[comp[s]] = s;
}

// Final signs: s_v = sig[v] * sig[r], r = ref[comp[v]] the vertex whose sign
// the reference's walk leaves unchanged at the start of v's part of the tree.
__global__ void k_kr_apply(int n, const int* __restrict__ comp, const int* __restrict__ ref,
                           const signed char* __restrict__ sig, float* __restrict__ nrm) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    if (sig[v] * sig[ref[comp[v]]] < 0) {
        nrm[v] = -nrm[v];
        nrm[n + v] = -nrm[n + v];
        nrm[2 * (size_t)n + v] = -nrm[2 * (size_t)n + v];
    }
}

__global__ void k_set_int(int* p, int v) { *p = v; }

// Device buffers of one spanning-forest computation over n vertices.
struct Forest {
    int* comp = nullptr;
    int* link = nullptr;
    int* link2 = nullptr;
    signed char* sig = nullptr;
    signed char* lpar = nullptr;
    signed char* lpar2 = nullptr;
    unsigned long long* best = nullptr;
    unsigned long long* first = nullptr;

    cudaError_t alloc(int n, cudaStream_t st) {
        cudaError_t e = cudaSuccess;
        auto A = [&](auto** p, size_t bytes) {
            if (e == cudaSuccess) e = cudaMallocAsync((void**)p, bytes, st);
        };
        A(&comp, sizeof(int) * n); A(&link, sizeof(int) * n); A(&link2, sizeof(int) * n);
        A(&sig, n); A(&lpar, n); A(&lpar2, n);
        A(&best, sizeof(unsigned long long) * n); A(&first, sizeof(unsigned long long) * n);
        return e;
    }
    void release(cudaStream_t st) {
        for (void* p : {(void*)comp, (void*)link, (void*)link2, (void*)sig, (void*)lpar, (void*)lpar2, (void*)best,
                        (void*)first})
            if (p) cudaFreeAsync(p, st);
    }
};

// Borůvka minimum spanning forest with sign parity.  act[0..E): order keys
// (rank << 32 | edge), the low half indexing ukey (u << bits | v) and sgn
// (+-1); the order keys are compacted in place as edges fall inside one
// component.  On return f.comp[v] is v's component representative, f.sig[v]
// the product of the edge signs on the forest path from the representative to
// v, and f.first[v] the order key of v's lightest edge.  msf (optional):
// msf[edge] = 1 for every forest edge.  ctr: device counters (kCtrFlag and
// kCtrMsf are used).  tmp / t_live: scratch for cub::DeviceSelect::If.
egt_status spanning_forest(int n, int E, int bits, const unsigned long long* ukey, unsigned long long* act,
                           const signed char* sgn, int* d_num, void* tmp, size_t t_live,
                           unsigned long long* ctr, Forest& f, unsigned char* msf, cudaStream_t st) {
    const unsigned TB = 256;
    auto G = [&](int64_t m) { return (unsigned)((m + TB - 1) / TB); };
    k_set_int<<<1, 1, 0, st>>>(d_num, E);
    EGT_LAUNCH_CHECK();
    k_init_comp<<<G(n), TB, 0, st>>>(n, f.comp, f.sig);
    EGT_LAUNCH_CHECK();
    if (E == 0) {  // every vertex is its own component
        EGT_CUDA_TRY(cudaMemsetAsync(f.first, 0xff, sizeof(unsigned long long) * n, st));
        return EGT_OK;
    }
    JoinsTwo live_op{ukey, f.comp, bits};
    // each round at least halves the non-trivial components; *d_num counts
    // the live edges at the head of act
    int live = E;  // *d_num, read back once per round (an upper bound until then)
    for (int round = 0;; round++) {
        if (round > 64) { set_error("orientation: spanning forest did not converge"); return EGT_ERR_CAP_EXCEEDED; }
        EGT_CUDA_TRY(cudaMemsetAsync(f.best, 0xff, sizeof(unsigned long long) * n, st));
        EGT_CUDA_TRY(cudaMemsetAsync(ctr + kCtrFlag, 0, sizeof(unsigned long long), st));
        k_select<<<G(live), TB, 0, st>>>(act, d_num, ukey, bits, f.comp, f.best);
        EGT_LAUNCH_CHECK();
        if (round == 0)  // every vertex's lightest edge: the tree roots come from these
            EGT_CUDA_TRY(cudaMemcpyAsync(f.first, f.best, sizeof(unsigned long long) * n, cudaMemcpyDeviceToDevice, st));
        k_hook<<<G(n), TB, 0, st>>>(ukey, sgn, n, bits, f.comp, f.sig, f.best, f.link, f.lpar, ctr, msf);
        EGT_LAUNCH_CHECK();
        unsigned long long any = 0;
        EGT_CUDA_TRY(cudaMemcpyAsync(&any, ctr + kCtrFlag, sizeof(any), cudaMemcpyDeviceToHost, st));
        EGT_CUDA_TRY(cudaMemcpyAsync(&live, d_num, sizeof(int), cudaMemcpyDeviceToHost, st));
        EGT_CUDA_TRY(cudaStreamSynchronize(st));  // live is now exact: the compaction below reads it
        if (!any) break;
        // pointer jumping over the hook forest, composing the sign parities
        for (int it = 0;; it++) {
            if (it > 64) { set_error("orientation: pointer jumping did not converge"); return EGT_ERR_CAP_EXCEEDED; }
            EGT_CUDA_TRY(cudaMemsetAsync(ctr + kCtrFlag, 0, sizeof(unsigned long long), st));
            k_jump<<<G(n), TB, 0, st>>>(f.link, f.lpar, n, f.link2, f.lpar2, ctr);
            EGT_LAUNCH_CHECK();
            std::swap(f.link, f.link2);
            std::swap(f.lpar, f.lpar2);
            unsigned long long ch = 0;
            EGT_CUDA_TRY(cudaMemcpyAsync(&ch, ctr + kCtrFlag, sizeof(ch), cudaMemcpyDeviceToHost, st));
            EGT_CUDA_TRY(cudaStreamSynchronize(st));
            if (!ch) break;
        }
        k_relabel<<<G(n), TB, 0, st>>>(n, f.link, f.lpar, f.comp, f.sig);
        EGT_LAUNCH_CHECK();
        // drop the edges that now lie inside one component
        EGT_CUDA_TRY(cub::DeviceSelect::If(tmp, t_live, act, d_num, live, live_op, st));
    }
    return EGT_OK;
}

}  // namespace

egt_status run_orient(egt_handle* h) {
    cudaStream_t st = h->stream;
    const int n = (int)h->n;
    int64_t nnz = 0;
    EGT_TRY(csr_nnz(h, &nnz));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[10], st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrMsf, 0, 2 * sizeof(unsigned long long), st));
    if (nnz == 0 || n < 2) {
        EGT_CUDA_TRY(cudaEventRecord(h->ev[11], st));
        return EGT_OK;
    }
    int bits = 1;
    while ((1ll << bits) < (int64_t)n) bits++;
    const unsigned TB = 256;
    auto G = [&](int64_t m) { return (unsigned)((m + TB - 1) / TB); };
    // 1. undirected edge keys u*2^bits+v (u < v), sorted (key order = the
    // reference's hash order), first copies kept in place.  The two halves of
    // the sort's double buffer are the only edge-sized buffers: after the
    // sort one holds the edges, the other their order keys.
    unsigned long long *bufA = nullptr, *bufB = nullptr;
    unsigned char* flag = nullptr;
    int* d_num = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&bufA, sizeof(unsigned long long) * nnz, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&bufB, sizeof(unsigned long long) * nnz, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&flag, nnz, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&d_num, sizeof(int), st));
    k_edge_keys<<<G(n), TB, 0, st>>>(h->csr_off, h->csr_col, n, bits, bufA);
    EGT_LAUNCH_CHECK();
    cub::DoubleBuffer<unsigned long long> keys(bufA, bufB);
    size_t t_sort = 0, t_flag = 0, t_live = 0;
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, t_sort, keys, (int)nnz, 0, 2 * bits, st));
    EGT_CUDA_TRY(cub::DeviceSelect::Flagged(nullptr, t_flag, bufA, flag, d_num, (int)nnz, st));
    JoinsTwo live_op{nullptr, nullptr, bits};
    EGT_CUDA_TRY(cub::DeviceSelect::If(nullptr, t_live, bufA, d_num, (int)nnz, live_op, st));
    void* tmp = nullptr;
    EGT_TRY(scratch_reserve(h, std::max(std::max(t_sort, t_flag), t_live), &tmp));
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp, t_sort, keys, (int)nnz, 0, 2 * bits, st));
    unsigned long long* ukey = keys.Current();
    unsigned long long* act = keys.Alternate();
    k_first_copy<<<G(nnz), TB, 0, st>>>(ukey, nnz, bits, flag);
    EGT_LAUNCH_CHECK();
    EGT_CUDA_TRY(cub::DeviceSelect::Flagged(tmp, t_flag, ukey, flag, d_num, (int)nnz, st));
    int E = 0;
    EGT_CUDA_TRY(cudaMemcpyAsync(&E, d_num, sizeof(int), cudaMemcpyDeviceToHost, st));
    EGT_CUDA_TRY(cudaStreamSynchronize(st));
    // ukey now holds the E unique edges in ascending key order
    signed char* sgn = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&sgn, std::max(E, 1), st));
    Forest f;
    EGT_CUDA_TRY(f.alloc(n, st));
    egt_status status = EGT_OK;
    if (E > 0) {
        k_edge_init<<<G(E), TB, 0, st>>>(ukey, E, bits, h->nrm, n, act, sgn);
        EGT_LAUNCH_CHECK();
        // 2. Borůvka rounds
        status = spanning_forest(n, E, bits, ukey, act, sgn, d_num, tmp, t_live, h->d_counters, f, nullptr, st);
        if (status == EGT_OK) {
            // 3. roots (first vertex of each tree's lightest edge) and signs
            EGT_CUDA_TRY(cudaMemsetAsync(f.best, 0xff, sizeof(unsigned long long) * n, st));
            k_roots<<<G(n), TB, 0, st>>>(n, f.comp, f.first, f.best);
            EGT_LAUNCH_CHECK();
            k_apply<<<G(n), TB, 0, st>>>(n, bits, f.comp, f.sig, f.best, ukey, h->nrm, h->d_counters);
            EGT_LAUNCH_CHECK();
        }
    }
    cudaFreeAsync(bufA, st); cudaFreeAsync(bufB, st); cudaFreeAsync(flag, st); cudaFreeAsync(d_num, st);
    cudaFreeAsync(sgn, st);
    f.release(st);
    EGT_CUDA_TRY(cudaEventRecord(h->ev[11], st));
    return status;
}

// orient_kruskal (MST.cpp:399-423) with Graph::kruskalMST (:297-376),
// DisjointSets (:185-229) and orientSpanningTree (:262-279), the reference's
// CPU orienter, on the GPU.  The reference keeps each undirected list edge
// once, sorts the edges by (weight, u, v) with weight max(0, 1 - |n_u . n_v|)
// in double, runs Kruskal with a union-find (union by rank, the second root
// winning ties), and walks every tree depth-first from its union-find root,
// negating a child whose float dot product with its (final) parent normal is
// negative.  Here:
//   1. the edge keys are sorted and deduplicated, the weights computed with
//      the reference's rounding, and the edges ranked by a stable sort on the
//      weight bits -- the reference's (weight, u, v) order;
//   2. Borůvka over that total order gives the same (unique) forest, with each
//      vertex's sign parity relative to its component;
//   3. the union-find roots depend on the order of the unions, so the forest
//      edges are replayed on the host in Kruskal order (n - components unions,
//      no sorting, no edge scan) with the reference's rank rule;
//   4. along a tree path the walk's rule multiplies the edge signs, except
//      across an edge whose dot product is exactly zero: the child is then
//      left as it is and its subtree follows from it.  So each vertex's sign is
//      its parity relative to the start of its part of the tree: the root, or
//      the child end of the last zero edge above it.  Parts are found (only
//      when zero edges exist) by a second forest pass without the zero edges
//      and a walk over the few zero edges on the host.
// knn: n rows of k ints (device), the first k_use of each read; nrm: [3n] SoA
// normals (device), in place.
egt_status run_orient_kruskal(const int* knn, float* nrm, int n, int k, int k_use, cudaStream_t st) {
    if (n < 2 || k_use < 1) return EGT_OK;
    const int64_t slots = (int64_t)n * k_use;
    if (slots > INT32_MAX) { set_error("orient_kruskal: n * k_use exceeds 2^31 - 1 list entries"); return EGT_ERR_CAP_EXCEEDED; }
    int bits = 1;
    while ((1ll << bits) < (int64_t)n) bits++;
    const unsigned TB = 256;
    auto G = [&](int64_t m) { return (unsigned)((m + TB - 1) / TB); };
    std::vector<void*> owned;
    auto D = [&](auto** p, size_t bytes) {
        const cudaError_t e = cudaMallocAsync((void**)p, std::max<size_t>(bytes, 16), st);
        if (e == cudaSuccess) owned.push_back((void*)*p);
        return e;
    };
    struct Releaser {
        std::vector<void*>& v;
        cudaStream_t st;
        ~Releaser() { for (void* p : v) cudaFreeAsync(p, st); }
    } releaser{owned, st};
    unsigned long long *ctr = nullptr, *bufA = nullptr, *bufB = nullptr;
    unsigned char* flag = nullptr;
    int* d_num = nullptr;
    EGT_CUDA_TRY(D(&ctr, sizeof(unsigned long long) * kCtrWords));
    EGT_CUDA_TRY(D(&bufA, sizeof(unsigned long long) * slots));
    EGT_CUDA_TRY(D(&bufB, sizeof(unsigned long long) * slots));
    EGT_CUDA_TRY(D(&flag, slots));
    EGT_CUDA_TRY(D(&d_num, sizeof(int)));
    EGT_CUDA_TRY(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long) * kCtrWords, st));
    k_kr_keys<<<G(slots), TB, 0, st>>>(knn, n, k, k_use, bits, bufA, ctr);
    EGT_LAUNCH_CHECK();
    // 1. unique edges in (u, v) order
    cub::DoubleBuffer<unsigned long long> keys(bufA, bufB);
    size_t t_sort = 0, t_flag = 0;
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, t_sort, keys, (int)slots, 0, 2 * bits, st));
    EGT_CUDA_TRY(cub::DeviceSelect::Flagged(nullptr, t_flag, bufA, flag, d_num, (int)slots, st));
    void* tmp = nullptr;
    EGT_CUDA_TRY(D(&tmp, std::max(t_sort, t_flag)));
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp, t_sort, keys, (int)slots, 0, 2 * bits, st));
    unsigned long long* ukey = keys.Current();
    unsigned long long* act = keys.Alternate();
    k_first_copy<<<G(slots), TB, 0, st>>>(ukey, slots, bits, flag);
    EGT_LAUNCH_CHECK();
    EGT_CUDA_TRY(cub::DeviceSelect::Flagged(tmp, t_flag, ukey, flag, d_num, (int)slots, st));
    int E = 0;
    unsigned long long bad = 0;
    EGT_CUDA_TRY(cudaMemcpyAsync(&E, d_num, sizeof(int), cudaMemcpyDeviceToHost, st));
    EGT_CUDA_TRY(cudaMemcpyAsync(&bad, ctr + kCtrFlag, sizeof(bad), cudaMemcpyDeviceToHost, st));
    EGT_CUDA_TRY(cudaStreamSynchronize(st));
    if (bad) { set_error("orient_kruskal: a list entry is >= n"); return EGT_ERR_ARG; }
    if (E == 0) return EGT_OK;
    // weights, signs, and the rank of every edge in (weight, u, v) order
    unsigned long long *wkey = nullptr, *wkey2 = nullptr;
    int *eidx = nullptr, *order = nullptr;
    signed char* sgn = nullptr;
    unsigned char *zero = nullptr, *msf = nullptr;
    EGT_CUDA_TRY(D(&wkey, sizeof(unsigned long long) * E));
    EGT_CUDA_TRY(D(&wkey2, sizeof(unsigned long long) * E));
    EGT_CUDA_TRY(D(&eidx, sizeof(int) * E));
    EGT_CUDA_TRY(D(&order, sizeof(int) * E));
    EGT_CUDA_TRY(D(&sgn, E));
    EGT_CUDA_TRY(D(&zero, E));
    EGT_CUDA_TRY(D(&msf, E));
    k_kr_weights<<<G(E), TB, 0, st>>>(ukey, E, bits, nrm, n, wkey, eidx, sgn, zero);
    EGT_LAUNCH_CHECK();
    unsigned long long *vkey = nullptr, *okey = nullptr, *sel = nullptr;
    EGT_CUDA_TRY(D(&vkey, sizeof(unsigned long long) * E));
    EGT_CUDA_TRY(D(&okey, sizeof(unsigned long long) * E));
    EGT_CUDA_TRY(D(&sel, sizeof(unsigned long long) * E));
    unsigned char *f1 = nullptr, *f2 = nullptr, *f3 = nullptr;
    EGT_CUDA_TRY(D(&f1, E));
    EGT_CUDA_TRY(D(&f2, E));
    EGT_CUDA_TRY(D(&f3, E));
    size_t t_pairs = 0, t_live = 0, t_sel = 0;
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, t_pairs, wkey, wkey2, eidx, order, E, 0, 64, st));
    JoinsTwo probe{nullptr, nullptr, bits};
    EGT_CUDA_TRY(cub::DeviceSelect::If(nullptr, t_live, act, d_num, E, probe, st));
    EGT_CUDA_TRY(cub::DeviceSelect::Flagged(nullptr, t_sel, vkey, f1, sel, d_num, E, st));
    void* tmp2 = nullptr;
    EGT_CUDA_TRY(D(&tmp2, std::max(std::max(t_pairs, t_live), t_sel)));
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp2, t_pairs, wkey, wkey2, eidx, order, E, 0, 64, st));
    k_kr_rank<<<G(E), TB, 0, st>>>(order, E, act);
    EGT_LAUNCH_CHECK();
    EGT_CUDA_TRY(cudaMemsetAsync(msf, 0, E, st));
    // 2. the minimum spanning forest for that order, with sign parities
    Forest f;
    struct ForestReleaser {
        Forest& f;
        cudaStream_t st;
        ~ForestReleaser() { f.release(st); }
    } fr{f, st};
    EGT_CUDA_TRY(f.alloc(n, st));
    EGT_TRY(spanning_forest(n, E, bits, ukey, act, sgn, d_num, tmp2, t_live, ctr, f, msf, st));
    // forest edges in Kruskal order, and the zero-dot ones among them
    k_kr_forest_lists<<<G(E), TB, 0, st>>>(order, E, ukey, msf, zero, vkey, okey, f1, f2, f3);
    EGT_LAUNCH_CHECK();
    int m = 0;
    EGT_CUDA_TRY(cub::DeviceSelect::Flagged(tmp2, t_sel, vkey, f1, sel, d_num, E, st));
    EGT_CUDA_TRY(cudaMemcpyAsync(&m, d_num, sizeof(int), cudaMemcpyDeviceToHost, st));
    EGT_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<unsigned long long> tree((size_t)m);
    if (m) EGT_CUDA_TRY(cudaMemcpyAsync(tree.data(), sel, sizeof(unsigned long long) * m, cudaMemcpyDeviceToHost, st));
    EGT_CUDA_TRY(cudaStreamSynchronize(st));
    // 3. the reference's union-find, replayed over the forest edges in order
    // (union by rank, the second root winning ties; path halving in place of
    // the reference's full compression, which changes no root or rank; the
    // next edges' entries are prefetched, the accesses being random)
    const unsigned long long mask = (1ull << bits) - 1ull;
    std::vector<int> par((size_t)n);
    std::vector<unsigned char> rnk((size_t)n, 0);
    std::iota(par.begin(), par.end(), 0);
    auto find = [&](int x) {
        while (par[x] != x) {
            par[x] = par[par[x]];
            x = par[x];
        }
        return x;
    };
    constexpr size_t kAhead = 16;
    for (size_t i = 0; i < tree.size(); i++) {
        if (i + kAhead < tree.size()) {
            const unsigned long long t2 = tree[i + kAhead];
            __builtin_prefetch(&par[(int)(t2 >> bits)]);
            __builtin_prefetch(&par[(int)(t2 & mask)]);
        }
        const unsigned long long t = tree[i];
        const int a = find((int)(t >> bits)), b = find((int)(t & mask));
        if (a == b) continue;  // cannot happen for a forest; kept for safety
        if (rnk[a] > rnk[b]) par[b] = a;
        else par[a] = b;
        if (rnk[a] == rnk[b]) rnk[b]++;
    }
    // where each tree's walk starts: its union-find root (a root is a vertex
    // that is its own parent)
    std::vector<int> starts;
    // 4. zero-dot forest edges split the trees into parts
    int z = 0;
    EGT_CUDA_TRY(cub::DeviceSelect::Flagged(tmp2, t_sel, vkey, f3, sel, d_num, E, st));
    EGT_CUDA_TRY(cudaMemcpyAsync(&z, d_num, sizeof(int), cudaMemcpyDeviceToHost, st));
    EGT_CUDA_TRY(cudaStreamSynchronize(st));
    const int* comp_for_sign = f.comp;
    const signed char* sig_for_sign = f.sig;
    Forest g;
    struct ForestReleaser gr{g, st};
    if (z == 0) {
        for (int r = 0; r < n; r++)
            if (par[r] == r) starts.push_back(r);
    } else {
        std::vector<unsigned long long> zedges((size_t)z);
        EGT_CUDA_TRY(cudaMemcpyAsync(zedges.data(), sel, sizeof(unsigned long long) * z, cudaMemcpyDeviceToHost, st));
        EGT_CUDA_TRY(cudaStreamSynchronize(st));
        // parts: the forest without its zero edges
        int e2 = 0;
        EGT_CUDA_TRY(cub::DeviceSelect::Flagged(tmp2, t_sel, okey, f2, sel, d_num, E, st));
        EGT_CUDA_TRY(cudaMemcpyAsync(&e2, d_num, sizeof(int), cudaMemcpyDeviceToHost, st));
        EGT_CUDA_TRY(cudaStreamSynchronize(st));
        EGT_CUDA_TRY(g.alloc(n, st));
        EGT_TRY(spanning_forest(n, e2, bits, ukey, sel, sgn, d_num, tmp2, t_live, ctr, g, nullptr, st));
        std::vector<int> part((size_t)n);
        EGT_CUDA_TRY(cudaMemcpyAsync(part.data(), g.comp, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
        EGT_CUDA_TRY(cudaStreamSynchronize(st));
        // walk the parts from each tree's root part across the zero edges: the
        // part entered through zero edge (a, b) from a's side starts at b
        std::vector<std::vector<int>> by_part;
        std::vector<int> part_id((size_t)n, -1), start;
        auto pid = [&](int v) {
            int& p = part_id[part[v]];
            if (p < 0) { p = (int)start.size(); start.push_back(-1); by_part.emplace_back(); }
            return p;
        };
        for (int i = 0; i < z; i++) {
            const int a = (int)(zedges[i] >> bits), b = (int)(zedges[i] & mask);
            by_part[pid(a)].push_back(i);
            by_part[pid(b)].push_back(i);
        }
        std::vector<int> queue;
        for (int r = 0; r < n; r++) {
            if (par[r] != r) continue;
            const int p0 = part_id[part[r]];
            if (p0 < 0) {  // a tree without zero edges: one part
                starts.push_back(r);
                continue;
            }
            if (start[p0] >= 0) continue;
            start[p0] = r;
            queue.assign(1, p0);
            for (size_t qi = 0; qi < queue.size(); qi++) {
                const int p = queue[qi];
                for (int i : by_part[p]) {
                    const int a = (int)(zedges[i] >> bits), b = (int)(zedges[i] & mask);
                    const int pa = part_id[part[a]], pb = part_id[part[b]];
                    const int other = pa == p ? pb : pa;
                    if (start[other] >= 0) continue;
                    start[other] = pa == p ? b : a;
                    queue.push_back(other);
                }
            }
        }
        starts.insert(starts.end(), start.begin(), start.end());
        comp_for_sign = g.comp;
        sig_for_sign = g.sig;
    }
    // every vertex takes the sign parity relative to its part's start
    int *d_starts = nullptr, *d_ref = nullptr;
    const int ns = (int)starts.size();
    EGT_CUDA_TRY(D(&d_starts, sizeof(int) * ns));
    EGT_CUDA_TRY(D(&d_ref, sizeof(int) * n));
    EGT_CUDA_TRY(cudaMemcpyAsync(d_starts, starts.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st));
    k_kr_starts<<<G(ns), TB, 0, st>>>(d_starts, ns, comp_for_sign, d_ref);
    EGT_LAUNCH_CHECK();
    k_kr_apply<<<G(n), TB, 0, st>>>(n, comp_for_sign, d_ref, sig_for_sign, nrm);
    EGT_LAUNCH_CHECK();
    EGT_CUDA_TRY(cudaStreamSynchronize(st));  // host vectors above are read by pending copies
    return EGT_OK;
}

}  // namespace egt
