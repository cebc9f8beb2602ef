// Elliptic-Gabriel neighbour filter and CSR compaction.
//
// Reference: calculateEGG_GKNN (EGT_CUDA.cu:172-189) with the predicate
// isEllipicGabrielNeighbor_GKNN (EGT_CUDA.cu:136-170) and its frame helpers
// (EGT_CUDA.cu:34-134).  Entry j of a query's list is dropped when one of the
// closer listed neighbours j' < j lies strictly inside the ellipsoid centred on
// the midpoint of (p, q_j), with half-axis d = |q_j - p|/2 along q_j - p and
// alpha*d across.  The reference walks j downward and edits the list in place;
// because only indices >= j have been edited when entry j is tested, every
// test sees the unfiltered list, which is what this kernel does explicitly.
//
// One warp per query: lane l owns list slots l + 32*s.  Each lane builds the
// local frame of each of its slots once, then the warp broadcasts the closer
// neighbours one by one (shuffles) and every lane tests them against its
// slots.  The filtered list is written back in place (-1 for dropped entries,
// the reference's observable behaviour on GetKNNIndexesInPartitions), the kept
// count per row feeds a scan, and a second kernel packs the kept entries into
// CSR in list order for the Taubin and normals kernels.
#include <cub/cub.cuh>
#include "egt_internal.cuh"
#include "egt_filter.cuh"

namespace egt {
namespace {

constexpr int kWarps = 8;

// One query per group of G lanes (32 / G queries per warp).  Up to three
// slots per lane the registers are capped for four blocks per SM (the
// three-slot form spills a few registers and still runs 29 % faster than at
// three blocks).
template <int S, int G>
__global__ void __launch_bounds__(kWarps * 32, S <= 3 ? 4 : 1) k_egt(const float4* __restrict__ p4, int* __restrict__ lists,
                                                     int n, int k, float alpha, int* __restrict__ counts,
                                                     unsigned* __restrict__ tests_out) {
    constexpr int kPer = 32 / G;
    __shared__ float4 s_v[kWarps * kPer][G * S];
    const int lane = threadIdx.x & 31;
    const int g = (threadIdx.x >> 5) * kPer + lane / G;  // group in the block
    const int q0 = (blockIdx.x * kWarps + (threadIdx.x >> 5)) * kPer;
    if (q0 >= n) return;  // whole warps only
    const int q = q0 + lane / G;
    const bool active = q < n;
    unsigned tests = 0;
    const int cnt = egt_query<S, G>(p4, active ? p4[q] : make_float4(0.f, 0.f, 0.f, 0.f),
                                    lists + (size_t)(active ? q : 0) * k, k, alpha, lane, tests, s_v[g], active);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) tests += __shfl_xor_sync(0xffffffffu, tests, o);
    if (active && (lane & (G - 1)) == 0) {
        counts[q] = cnt;
        tests_out[q] = tests;
    }
}

// Sum of n counts into *out (one atomic per block).
__global__ void k_sum_counts(const unsigned* __restrict__ in, int n, unsigned long long* __restrict__ out) {
    __shared__ unsigned long long s_part[8];
    unsigned long long acc = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc += in[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s_part[w];
        if (t) atomicAdd(out, t);
    }
}

// Packs the kept entries of each row, in list order, into CSR columns.
template <int S>
__global__ void __launch_bounds__(kWarps * 32) k_compact(const int* __restrict__ lists, int n, int k,
                                                         const int* __restrict__ off, int* __restrict__ col) {
    const int lane = threadIdx.x & 31;
    const int q = blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (q >= n) return;
    int base = off[q];
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int t = lane + 32 * s;
        const int v = t < k ? lists[(size_t)q * k + t] : -1;
        const unsigned m = __ballot_sync(0xffffffffu, v >= 0);
        if (v >= 0) col[base + __popc(m & ((1u << lane) - 1u))] = v;
        base += __popc(m);
    }
}

__global__ void k_count_valid(const int* __restrict__ lists, int n, int k, int* __restrict__ counts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = 0;
    for (int j = 0; j < k; j++) c += lists[(size_t)i * k + j] >= 0;
    counts[i] = c;
}

template <int S, int G>
egt_status launch_egt(egt_handle* h, float alpha, int* counts, unsigned* tests) {
    const int per_block = kWarps * (32 / G);
    const unsigned B = (unsigned)((h->n + per_block - 1) / per_block);
    k_egt<S, G><<<B, kWarps * 32, 0, h->stream>>>(h->p4, h->lists, (int)h->n, h->k, alpha, counts, tests);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

template <int S>
egt_status launch_compact(egt_handle* h) {
    const unsigned G = (unsigned)((h->n + kWarps - 1) / kWarps);
    k_compact<S><<<G, kWarps * 32, 0, h->stream>>>(h->lists, (int)h->n, h->k, h->csr_off, h->csr_col);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

}  // namespace

// Builds the CSR view of the current lists.  counts [n+1] holds the kept
// entries per row (last element 0).  Columns are packed into a buffer of
// capacity n*k, so no host round trip is needed for the size; nnz is read back
// lazily (egt_get_timings / egt_get_csr).
static egt_status build_csr(egt_handle* h, int* counts) {
    cudaStream_t st = h->stream;
    const int64_t n = h->n;
    size_t cub_scan = 0;
    EGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, cub_scan, (int*)nullptr, (int*)nullptr, (int)(n + 1), st));
    void* tmp = nullptr;
    EGT_TRY(scratch_reserve(h, cub_scan, &tmp));
    if (!h->csr_off) EGT_CUDA_TRY(dev_alloc(h, &h->csr_off, sizeof(int) * (n + 1)));
    const int64_t cap = n * (int64_t)h->k;
    if (h->csr_cap < cap || !h->csr_col) {
        dev_free(h, h->csr_col);
        h->csr_col = nullptr;
        EGT_CUDA_TRY(dev_alloc(h, &h->csr_col, sizeof(int) * std::max<int64_t>(cap, 1)));
        h->csr_cap = std::max<int64_t>(cap, 1);
    }
    EGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, cub_scan, counts, h->csr_off, (int)(n + 1), st));
    const int k = h->k;
    if (k <= 32) EGT_TRY(launch_compact<1>(h));
    else if (k <= 64) EGT_TRY(launch_compact<2>(h));
    else if (k <= 128) EGT_TRY(launch_compact<4>(h));
    else EGT_TRY(launch_compact<8>(h));
    h->nnz = -1;  // known on the device; fetched on demand
    h->have_csr = true;
    h->csr_version++;
    return EGT_OK;
}

// Reads the CSR size back from the device (synchronises the stream).
egt_status csr_nnz(egt_handle* h, int64_t* out) {
    if (h->nnz < 0) {
        int v = 0;
        EGT_CUDA_TRY(cudaMemcpyAsync(&v, h->csr_off + h->n, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        EGT_CUDA_TRY(cudaStreamSynchronize(h->stream));
        h->nnz = v;
    }
    *out = h->nnz;
    return EGT_OK;
}

egt_status run_egt(egt_handle* h, float alpha) {
    if (!h->lists || h->k <= 0) { set_error("egt_filter: no neighbour lists (call egt_knn first)"); return EGT_ERR_STATE; }
    cudaStream_t st = h->stream;
    const int64_t n = h->n;
    int* counts = nullptr;
    unsigned* tests = nullptr;  // ellipsoid tests per query, summed for egt_get_timings
    EGT_CUDA_TRY(cudaMallocAsync((void**)&counts, sizeof(int) * (n + 1), st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&tests, sizeof(unsigned) * n, st));
    EGT_CUDA_TRY(cudaMemsetAsync(counts + n, 0, sizeof(int), st));
    EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrEgtTests, 0, sizeof(unsigned long long), st));
    EGT_CUDA_TRY(cudaEventRecord(h->ev[4], st));
    const int k = h->k;
    egt_status s;
    // lanes per query: 16 where a 32-lane round would leave half of it empty
    if (k <= 16) s = launch_egt<1, 16>(h, alpha, counts, tests);
    else if (k <= 32) s = launch_egt<1, 32>(h, alpha, counts, tests);
    else if (k <= 48) s = launch_egt<3, 16>(h, alpha, counts, tests);
    else if (k <= 64) s = launch_egt<2, 32>(h, alpha, counts, tests);
    else if (k <= 128) s = launch_egt<4, 32>(h, alpha, counts, tests);
    else s = launch_egt<8, 32>(h, alpha, counts, tests);
    EGT_CUDA_TRY(cudaEventRecord(h->ev[14], st));
    if (s == EGT_OK) s = build_csr(h, counts);
    EGT_CUDA_TRY(cudaEventRecord(h->ev[5], st));
    if (s == EGT_OK) {
        k_sum_counts<<<592, 256, 0, st>>>(tests, (int)n, h->d_counters + kCtrEgtTests);
        EGT_LAUNCH_CHECK();
    }
    cudaFreeAsync(counts, st);
    cudaFreeAsync(tests, st);
    return s;
}

// CSR of the unfiltered lists (used when Taubin/normals run without EGT).
egt_status ensure_csr(egt_handle* h) {
    if (h->have_csr) return EGT_OK;
    cudaStream_t st = h->stream;
    const int64_t n = h->n;
    int* counts = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&counts, sizeof(int) * (n + 1), st));
    EGT_CUDA_TRY(cudaMemsetAsync(counts + n, 0, sizeof(int), st));
    k_count_valid<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(h->lists, (int)n, h->k, counts);
    EGT_LAUNCH_CHECK();
    egt_status s = build_csr(h, counts);
    cudaFreeAsync(counts, st);
    return s;
}

}  // namespace egt
