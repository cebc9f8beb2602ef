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

__global__ void k_select(const unsigned long long* __restrict__ ukey, const unsigned long long* __restrict__ ckey,
                         int E, int bits, const int* __restrict__ comp, unsigned long long* __restrict__ best) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const unsigned long long k = ukey[e];
    const int u = (int)(k >> bits), v = (int)(k & ((1ull << bits) - 1ull));
    const int cu = comp[u], cv = comp[v];
    if (cu == cv) return;
    const unsigned long long c = ckey[e];
    atomicMin(&best[cu], c);
    atomicMin(&best[cv], c);
}

__global__ void k_hook(const unsigned long long* __restrict__ ukey, const signed char* __restrict__ sgn, int n,
                       int bits, const int* __restrict__ comp, const signed char* __restrict__ sig,
                       const unsigned long long* __restrict__ best, int* __restrict__ link,
                       signed char* __restrict__ lpar, unsigned char* __restrict__ msf,
                       unsigned long long* __restrict__ ctr) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    link[c] = c;
    lpar[c] = 1;
    if (comp[c] != c) return;
    const unsigned long long b = best[c];
    if (b == kNone) return;
    const int e = (int)(b & 0xffffffffull);
    const unsigned long long k = ukey[e];
    const int u = (int)(k >> bits), v = (int)(k & ((1ull << bits) - 1ull));
    const int x = comp[u] == c ? u : v;
    const int y = x == u ? v : u;
    const int c2 = comp[y];
    msf[e] = 1;
    atomicAdd(&ctr[kCtrFlag], 1ull);
    if (best[c2] == b && c < c2) return;  // mutual choice: the smaller representative stays a root
    link[c] = c2;
    lpar[c] = (signed char)(sig[x] * sgn[e] * sig[y]);
}

__global__ void k_jump(const int* __restrict__ link, const signed char* __restrict__ lpar, int n,
                       int* __restrict__ link2, signed char* __restrict__ lpar2, unsigned long long* __restrict__ ctr) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int l = link[c];
    const int ll = link[l];
    if (l != ll) {
        link2[c] = ll;
        lpar2[c] = (signed char)(lpar[c] * lpar[l]);
        atomicAdd(&ctr[kCtrFlag], 1ull);
    } else {
        link2[c] = l;
        lpar2[c] = lpar[c];
    }
}

__global__ void k_relabel(int n, const int* __restrict__ link, const signed char* __restrict__ lpar,
                          int* __restrict__ comp, signed char* __restrict__ sig) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int c = comp[v];
    comp[v] = link[c];
    sig[v] = (signed char)(sig[v] * lpar[c]);
}

__global__ void k_roots(const unsigned long long* __restrict__ ckey, const unsigned long long* __restrict__ ukey,
                        int E, int bits, const int* __restrict__ comp, unsigned long long* __restrict__ rootkey,
                        const unsigned char* __restrict__ msf, unsigned long long* __restrict__ ctr) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int u = (int)(ukey[e] >> bits);
    atomicMin(&rootkey[comp[u]], ckey[e]);
    if (msf[e]) atomicAdd(&ctr[kCtrMsf], 1ull);
}

__global__ void k_apply(int n, int bits, const int* __restrict__ comp, const signed char* __restrict__ sig,
                        const unsigned long long* __restrict__ rootkey, const unsigned long long* __restrict__ ukey,
                        float* __restrict__ nrm, unsigned long long* __restrict__ ctr) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int c = comp[v];
    const unsigned long long rk = rootkey[c];
    if (rk == kNone) return;  // no edge: keeps its unoriented normal
    const int e = (int)(rk & 0xffffffffull);
    const int R = (int)(ukey[e] >> bits);
    if (v == c) atomicAdd(&ctr[kCtrComps], 1ull);
    if (sig[v] * sig[R] < 0) {
        nrm[v] = -nrm[v];
        nrm[n + v] = -nrm[n + v];
        nrm[2 * (size_t)n + v] = -nrm[2 * (size_t)n + v];
    }
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
    // 1. undirected edge keys, sorted and unique (key order = the reference's hash order)
    unsigned long long *key = nullptr, *ukey = nullptr;
    int* d_num = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&key, sizeof(unsigned long long) * nnz, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&ukey, sizeof(unsigned long long) * nnz, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&d_num, sizeof(int), st));
    k_edge_keys<<<G(n), TB, 0, st>>>(h->csr_off, h->csr_col, n, bits, key);
    EGT_LAUNCH_CHECK();
    size_t t_sort = 0, t_uniq = 0;
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, t_sort, key, ukey, (int)nnz, 0, 2 * bits, st));
    EGT_CUDA_TRY(cub::DeviceSelect::Unique(nullptr, t_uniq, ukey, key, d_num, (int)nnz, st));
    void* tmp = nullptr;
    EGT_TRY(scratch_reserve(h, std::max(t_sort, t_uniq), &tmp));
    EGT_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp, t_sort, key, ukey, (int)nnz, 0, 2 * bits, st));
    EGT_CUDA_TRY(cub::DeviceSelect::Unique(tmp, t_uniq, ukey, key, d_num, (int)nnz, st));
    int E = 0;
    EGT_CUDA_TRY(cudaMemcpyAsync(&E, d_num, sizeof(int), cudaMemcpyDeviceToHost, st));
    unsigned long long last = 0;
    EGT_CUDA_TRY(cudaStreamSynchronize(st));
    if (E > 0) {
        EGT_CUDA_TRY(cudaMemcpy(&last, key + (E - 1), sizeof(last), cudaMemcpyDeviceToHost));
        if (last == (1ull << (2 * bits)) - 1ull) E--;  // self-loop sentinel
    }
    // key now holds the E unique edges in ascending key order
    unsigned long long *ckey = nullptr, *best = nullptr;
    signed char *sgn = nullptr, *sig = nullptr, *lpar = nullptr, *lpar2 = nullptr;
    int *comp = nullptr, *link = nullptr, *link2 = nullptr;
    unsigned char* msf = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&ckey, sizeof(unsigned long long) * std::max(E, 1), st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&sgn, std::max(E, 1), st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&msf, std::max(E, 1), st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&best, sizeof(unsigned long long) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&comp, sizeof(int) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&link, sizeof(int) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&link2, sizeof(int) * n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&sig, n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&lpar, n, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&lpar2, n, st));
    egt_status status = EGT_OK;
    if (E > 0) {
        k_edge_init<<<G(E), TB, 0, st>>>(key, E, bits, h->nrm, n, ckey, sgn);
        EGT_LAUNCH_CHECK();
        EGT_CUDA_TRY(cudaMemsetAsync(msf, 0, E, st));
        k_init_comp<<<G(n), TB, 0, st>>>(n, comp, sig);
        EGT_LAUNCH_CHECK();
        // 2. Borůvka rounds (each at least halves the non-trivial components)
        int round = 0;
        for (;; round++) {
            if (round > 64) { set_error("orientation: spanning forest did not converge"); status = EGT_ERR_CAP_EXCEEDED; break; }
            EGT_CUDA_TRY(cudaMemsetAsync(best, 0xff, sizeof(unsigned long long) * n, st));
            EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrFlag, 0, sizeof(unsigned long long), st));
            k_select<<<G(E), TB, 0, st>>>(key, ckey, E, bits, comp, best);
            EGT_LAUNCH_CHECK();
            k_hook<<<G(n), TB, 0, st>>>(key, sgn, n, bits, comp, sig, best, link, lpar, msf, h->d_counters);
            EGT_LAUNCH_CHECK();
            unsigned long long any = 0;
            EGT_CUDA_TRY(cudaMemcpyAsync(&any, h->d_counters + kCtrFlag, sizeof(any), cudaMemcpyDeviceToHost, st));
            EGT_CUDA_TRY(cudaStreamSynchronize(st));
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
        }
        if (status == EGT_OK) {
            // 3. roots (first vertex of each tree's lightest edge) and signs
            EGT_CUDA_TRY(cudaMemsetAsync(best, 0xff, sizeof(unsigned long long) * n, st));
            k_roots<<<G(E), TB, 0, st>>>(ckey, key, E, bits, comp, best, msf, h->d_counters);
            EGT_LAUNCH_CHECK();
            k_apply<<<G(n), TB, 0, st>>>(n, bits, comp, sig, best, key, h->nrm, h->d_counters);
            EGT_LAUNCH_CHECK();
        }
    }
    cudaFreeAsync(key, st); cudaFreeAsync(ukey, st); cudaFreeAsync(d_num, st);
    cudaFreeAsync(ckey, st); cudaFreeAsync(sgn, st); cudaFreeAsync(msf, st); cudaFreeAsync(best, st);
    cudaFreeAsync(comp, st); cudaFreeAsync(link, st); cudaFreeAsync(link2, st);
    cudaFreeAsync(sig, st); cudaFreeAsync(lpar, st); cudaFreeAsync(lpar2, st);
    EGT_CUDA_TRY(cudaEventRecord(h->ev[11], st));
    return status;
}

}  // namespace egt
