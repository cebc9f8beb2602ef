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
                       signed char* __restrict__ lpar, unsigned long long* __restrict__ ctr) {
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
    unsigned long long *best = nullptr, *first = nullptr;
    signed char *sgn = nullptr, *sig = nullptr, *lpar = nullptr, *lpar2 = nullptr;
    int *comp = nullptr, *link = nullptr, *link2 = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&sgn, std::max(E, 1), st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&best, sizeof(unsigned long long) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&first, sizeof(unsigned long long) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&comp, sizeof(int) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&link, sizeof(int) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&link2, sizeof(int) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&sig, n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&lpar, n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&lpar2, n, st));
    egt_status status = EGT_OK;
    if (E > 0) {
        k_edge_init<<<G(E), TB, 0, st>>>(ukey, E, bits, h->nrm, n, act, sgn);
        EGT_LAUNCH_CHECK();
        k_init_comp<<<G(n), TB, 0, st>>>(n, comp, sig);
        EGT_LAUNCH_CHECK();
        live_op.ukey = ukey;
        live_op.comp = comp;
        // 2. Borůvka rounds (each at least halves the non-trivial components);
        // *d_num counts the live edges at the head of act
        int live = E;  // *d_num, read back once per round (an upper bound until then)
        for (int round = 0;; round++) {
            if (round > 64) { set_error("orientation: spanning forest did not converge"); status = EGT_ERR_CAP_EXCEEDED; break; }
            EGT_CUDA_TRY(cudaMemsetAsync(best, 0xff, sizeof(unsigned long long) * n, st));
            EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrFlag, 0, sizeof(unsigned long long), st));
            k_select<<<G(live), TB, 0, st>>>(act, d_num, ukey, bits, comp, best);
            EGT_LAUNCH_CHECK();
            if (round == 0)  // every vertex's lightest edge: the tree roots come from these
                EGT_CUDA_TRY(cudaMemcpyAsync(first, best, sizeof(unsigned long long) * n, cudaMemcpyDeviceToDevice, st));
            k_hook<<<G(n), TB, 0, st>>>(ukey, sgn, n, bits, comp, sig, best, link, lpar, h->d_counters);
            EGT_LAUNCH_CHECK();
            unsigned long long any = 0;
            EGT_CUDA_TRY(cudaMemcpyAsync(&any, h->d_counters + kCtrFlag, sizeof(any), cudaMemcpyDeviceToHost, st));
            EGT_CUDA_TRY(cudaMemcpyAsync(&live, d_num, sizeof(int), cudaMemcpyDeviceToHost, st));
            EGT_CUDA_TRY(cudaStreamSynchronize(st));  // live is now exact: the compaction below reads it
            if (!any) break;
            // pointer jumping over the hook forest, composing the sign parities
            for (int it = 0;; it++) {
                if (it > 64) { set_error("orientation: pointer jumping did not converge"); status = EGT_ERR_CAP_EXCEEDED; break; }
                EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrFlag, 0, sizeof(unsigned long long), st));
                k_jump<<<G(n), TB, 0, st>>>(link, lpar, n, link2, lpar2, h->d_counters);
                EGT_LAUNCH_CHECK();
                std::swap(link, link2);
                std::swap(lpar, lpar2);
                unsigned long long ch = 0;
                EGT_CUDA_TRY(cudaMemcpyAsync(&ch, h->d_counters + kCtrFlag, sizeof(ch), cudaMemcpyDeviceToHost, st));
                EGT_CUDA_TRY(cudaStreamSynchronize(st));
                if (!ch) break;
            }
            if (status != EGT_OK) break;
            k_relabel<<<G(n), TB, 0, st>>>(n, link, lpar, comp, sig);
            EGT_LAUNCH_CHECK();
            // drop the edges that now lie inside one component
            EGT_CUDA_TRY(cub::DeviceSelect::If(tmp, t_live, act, d_num, live, live_op, st));
        }
        if (status == EGT_OK) {
            // 3. roots (first vertex of each tree's lightest edge) and signs
            EGT_CUDA_TRY(cudaMemsetAsync(best, 0xff, sizeof(unsigned long long) * n, st));
            k_roots<<<G(n), TB, 0, st>>>(n, comp, first, best);
            EGT_LAUNCH_CHECK();
            k_apply<<<G(n), TB, 0, st>>>(n, bits, comp, sig, best, ukey, h->nrm, h->d_counters);
            EGT_LAUNCH_CHECK();
        }
    }
    cudaFreeAsync(bufA, st); cudaFreeAsync(bufB, st); cudaFreeAsync(flag, st); cudaFreeAsync(d_num, st);
    cudaFreeAsync(sgn, st); cudaFreeAsync(best, st); cudaFreeAsync(first, st);
    cudaFreeAsync(comp, st); cudaFreeAsync(link, st); cudaFreeAsync(link2, st);
    cudaFreeAsync(sig, st); cudaFreeAsync(lpar, st); cudaFreeAsync(lpar2, st);
    EGT_CUDA_TRY(cudaEventRecord(h->ev[11], st));
    return status;
}

}  // namespace egt
