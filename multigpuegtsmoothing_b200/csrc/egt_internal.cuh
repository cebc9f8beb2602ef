// Internal definitions shared by the CUDA translation units of libegt_b200.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "egt_b200.h"

namespace egt {

// ---------------------------------------------------------------------------
// Error plumbing: every CUDA call is checked and mapped to an egt_status.
void set_error(const std::string& msg);
std::string cuda_msg(cudaError_t e, const char* what, const char* file, int line);

#define EGT_CUDA_TRY(call)                                                         \
    do {                                                                           \
        cudaError_t e__ = (call);                                                  \
        if (e__ != cudaSuccess) {                                                  \
            ::egt::set_error(::egt::cuda_msg(e__, #call, __FILE__, __LINE__));      \
            return e__ == cudaErrorMemoryAllocation ? EGT_ERR_NOMEM : EGT_ERR_CUDA;\
        }                                                                          \
    } while (0)

// Every kernel launch site is followed by EGT_LAUNCH_CHECK(), which also counts
// the launch (egt_kernel_launches()).
void count_launch();
#define EGT_LAUNCH_CHECK()        \
    do {                          \
        ::egt::count_launch();    \
        EGT_CUDA_TRY(cudaGetLastError()); \
    } while (0)

#define EGT_TRY(st)                          \
    do {                                     \
        egt_status s__ = (st);               \
        if (s__ != EGT_OK) return s__;       \
    } while (0)

// ---------------------------------------------------------------------------
// Device rounding shapes.  The reference is built with nvcc's default
// --fmad=true; these helpers spell out the fused multiply-adds that compiler
// forms for each expression (identified black-box, see oracle/fp_shapes.h),
// so results are bit-identical to the reference whatever the surrounding code.
__device__ __forceinline__ float fs_dist3(float ax, float ay, float az, float bx, float by, float bz) {
    float dx = __fsub_rn(ax, bx), dy = __fsub_rn(ay, by), dz = __fsub_rn(az, bz);
    return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}
__device__ __forceinline__ float fs_sq3(float x, float y, float z) {
    return __fmaf_rn(z, z, __fmaf_rn(x, x, __fmul_rn(y, y)));
}
__device__ __forceinline__ float fs_dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return __fmaf_rn(az, bz, __fmaf_rn(ax, bx, __fmul_rn(ay, by)));
}
__device__ __forceinline__ float fs_face_lo(float x, float xmin, float f, float h) {
    return __fmaf_rn(-f, h, __fsub_rn(x, xmin));
}
__device__ __forceinline__ float fs_face_hi(float x, float xmin, float f, float h) {
    return __fmaf_rn(f, h, __fsub_rn(xmin, x));
}
__device__ __forceinline__ float fs_cross1(float u2, float v3, float v2, float u3) {
    return __fmaf_rn(u2, v3, -__fmul_rn(v2, u3));
}
__device__ __forceinline__ float fs_affine(float a1, float a2, float a3, float a4, float x, float y, float z) {
    return __fadd_rn(__fmaf_rn(a3, z, __fmaf_rn(a1, x, __fmul_rn(a2, y))), a4);
}
__device__ __forceinline__ float fs_ellipsoid(float x, float y, float z, float aa) {
    return __fadd_rn(__fmaf_rn(x, x, __fdiv_rn(__fmul_rn(y, y), aa)), __fdiv_rn(__fmul_rn(z, z), aa));
}
__device__ __forceinline__ float fs_lin2_add(float c, float a, float s, float b) {
    return __fmaf_rn(c, a, __fmul_rn(s, b));
}
__device__ __forceinline__ float fs_lin2_sub(float s, float a, float c, float b) {
    return __fmaf_rn(s, a, -__fmul_rn(c, b));
}
__device__ __forceinline__ float fs_sq2(float u, float v) { return __fmaf_rn(u, u, __fmul_rn(v, v)); }

// Cell coordinate of a normalised coordinate (GridKNNCuda.cu:74-88, :649-653).
__device__ __forceinline__ int cell_coord(float x, float a, float b, int B) {
    return (int)__fmul_rn(__fdiv_rn(__fsub_rn(x, a), __fsub_rn(b, a)), (float)B);
}

// ---------------------------------------------------------------------------
// Normalisation parameters, computed on the device (no host round trip).
struct NormParams {
    float mn, mx;      // scalar cube (GridKNNCuda.cu:1042-1071)
    float a, b;        // unit cube with eps: a = -eps, b = 1 + eps
    float thres;       // (thres / (mx - mn))^2 (GridKNNCuda.cu:2324-2325)
    int n;
};

constexpr int kMaxLevels = 8;  // levels 0..7 (B = 1024 .. 8) are searched

// Layout of egt_handle::d_counters (unsigned long long words).
constexpr int kCtrWords = 64;
constexpr int kCtrNcells = 0;     // [0..7]  occupied cells per level (int in a u64 slot)
constexpr int kCtrExtents = 16;   // [16..18] six packed u32 min/max words
constexpr int kCtrInvalid = 24;   // invalid queries of the last kNN
constexpr int kCtrMaxLevel = 25;  // deepest level reached
constexpr int kCtrNnz = 26;       // EGT kept neighbours
constexpr int kCtrFlag = 27;      // generic loop flag
constexpr int kCtrNormFallback = 28;  // normals re-solved in FP64
constexpr int kCtrMsf = 29;       // spanning-forest edges
constexpr int kCtrComps = 30;     // orientation components
constexpr int kCtrMaxPop = 32;    // [32..39] largest cell population per level
constexpr int kCtrBoxTried = 40;  // learned kNN: queries that ran a box search
constexpr int kCtrCertified = 41; // learned kNN: certified box results
constexpr int kCtrExactRerun = 42;  // kNN queries re-searched with the exact insertion rule (ties)
constexpr int kCtrWork = 43;        // work queue of the persistent kNN kernels (reset with 42)
constexpr int kCtrEvals = 44;       // plain kNN: candidate distances evaluated (reset with 42)
constexpr int kCtrEgtTests = 45;    // EGT filter: ellipsoid tests of the last filter run
constexpr int kCtrSpillTiles = 46;  // Taubin tiles that gather from global memory (too large to stage)
constexpr int kCtrSelFallback = 48; // queries the selection kNN could not certify (the ring search ran them)
constexpr int kCtrTileUnits = 49;    // cell-tile kNN: units (level, cell) to search
constexpr int kCtrTileWork = 50;     // cell-tile kNN: next unit to claim
constexpr int kCtrTileRingWork = 51; // cell-tile kNN: work counter of the ring search over its leftovers
constexpr int kCtrTileQ = 52;        // cell-tile kNN: queries compacted by unit
constexpr int kCtrTileRing2 = 55;    // cell-tile kNN: queries it could not certify (the ring search ran them)
constexpr int kCtrTileRingWork1 = 56; // cell-tile kNN: next unselected query for the ring search in the tile kernel

// One level of the cell hierarchy.  Cells are sorted by key
// x + y*B + z*B^2; a row is the set of occupied cells sharing (y, z).
struct LevelDev {
    int B = 0;
    int ncells = 0;
    int* order = nullptr;      // [n] sorted indices grouped by cell (level 0: identity, not stored)
    int* cell_start = nullptr; // [ncells+1] offsets into order
    int* cell_x = nullptr;     // [ncells] x coordinate of each cell
    int2* row_range = nullptr; // [B*B] [first, last) cell of each (y,z) row
};

struct Scratch {
    void* ptr = nullptr;
    size_t bytes = 0;
};

}  // namespace egt

struct egt_handle {
    egt_config cfg{};
    int64_t n = 0;
    int k = 0;
    bool is_mesh = false;
    cudaStream_t stream = nullptr;
    // positions
    float4* p4 = nullptr;        // [n] sorted, normalised (x,y,z,0)
    float4* p4b = nullptr;       // [n] ping-pong buffer for Taubin
    float* x = nullptr;          // [n] SoA mirror for the KNNInterface views
    float* y = nullptr;
    float* z = nullptr;
    uint32_t* cell0 = nullptr;   // [n] packed level-0 cell coords x | y<<10 | z<<20
    int* perm = nullptr;         // [n] sorted -> original
    egt::NormParams* d_norm = nullptr;
    egt::NormParams norm{};      // host copy
    egt::LevelDev lv[egt::kMaxLevels];
    int levels_built = 0;
    // neighbourhoods
    int* lists = nullptr;        // [n*k] sorted-space lists
    float* kth = nullptr;        // [n] k-th distance per query (diagnostics / learned labels)
    uint8_t* qlevel = nullptr;   // [n] level at which each query stopped
    // learned search proposal
    uint8_t* pclass = nullptr;   // [n] proposed class per query
    bool maxpop_valid = false;   // counters[kCtrMaxPop..] match the current grid
    const egt_proposal* proposal = nullptr;  // attached for knn_mode == EGT_KNN_LEARNED
    bool last_knn_learned = false;
    void* tile_mem = nullptr;    // cell-tile kNN: query levels, unit bits, units, leftover queries
    size_t tile_bytes = 0;
    int* csr_off = nullptr;      // [n+1]
    int* csr_col = nullptr;      // [nnz]
    int64_t csr_cap = 0;
    int64_t nnz = 0;             // -1 while only the device knows it
    bool have_csr = false;
    // mesh
    uint32_t* tris = nullptr;    // [3t] sorted-space triangle corners
    int64_t t = 0;
    // normals
    float* nrm = nullptr;        // [3n] SoA sorted-space normals
    // device counters
    unsigned long long* d_counters = nullptr;  // [kCtrWords] device counters
    // Taubin working set in Morton order of the level-0 cells
    int* m_perm = nullptr;       // [n] Morton position -> sorted index
    int* m_inv = nullptr;        // [n] sorted index -> Morton position
    float4* m_p = nullptr;       // [n] positions (Morton order)
    float4* m_pb = nullptr;      // [n] ping-pong
    int* m_off = nullptr;        // [n+1]
    int* m_col = nullptr;        // [nnz]
    int64_t m_cap = 0;
    // per 256-row tile: distinct neighbour indices (stored at the tile's first
    // CSR offset) and, per CSR entry, its index into that list
    int* t_uni = nullptr;        // [tiles * 1024] point index of each staged slot
    uint32_t* t_loc = nullptr;   // [tiles * 1792] CSR entries' slots, three 10-bit slots per word, sliced by warp
    int* t_nu = nullptr;         // [tiles] staged slot count, -1 = tile not staged
    int* t_soff = nullptr;       // [tiles * 9] slice offsets into t_loc, then the table size
    int64_t t_tiles = 0;         // tiles the four tables above are sized for
    uint64_t csr_version = 0;    // bumped whenever the CSR is rebuilt
    uint64_t m_version = ~0ull;  // CSR version the Morton copy was built from
    // cached Taubin graph (2*iters half-steps) and the parameters it was built for
    cudaGraphExec_t taubin_exec = nullptr;
    int taubin_iters = -1;
    float taubin_lambda = 0.f, taubin_mu = 0.f;
    const void* taubin_key[8] = {};
    int taubin_mode = 0;         // 0: staged tiles, 1: direct gathers (chosen by the batch autotuner)
    int taubin_graph_mode = -1;  // mode the cached graph was captured with
    // batched clouds: per-point cloud id (sorted order), bits of the largest id
    const uint16_t* cloud_of = nullptr;
    int cloud_bits = 0;
    // timing
    cudaEvent_t ev[16] = {};
    egt_timings tm{};
    egt::Scratch scratch;
};

namespace egt {
// Handle buffers come from the device's stream-ordered memory pool (kept warm
// with a high release threshold), so creating and destroying providers
// repeatedly reuses memory instead of returning it to the driver.
template <typename T>
inline cudaError_t dev_alloc(egt_handle* h, T** p, size_t bytes) {
    return cudaMallocAsync(reinterpret_cast<void**>(p), bytes, h->stream);
}
inline void dev_free(egt_handle* h, void* p) {
    if (p) cudaFreeAsync(p, h->stream);
}
egt_status scratch_reserve(egt_handle* h, size_t bytes, void** out);
egt_status build_grid(egt_handle* h, const float* xyz_dev_aos, int levels);
egt_status set_threshold(egt_handle* h, float thres);
egt_status run_knn(egt_handle* h, int k);
egt_status run_knn_host(egt_handle* h, int k, int* host);
egt_status run_knn_query(egt_handle* h, const float* q_host, int64_t nq, int k, int* out_host, int64_t* invalid);
egt_status run_knn_learned(egt_handle* h, int k, const egt_proposal* p);
int proposal_k(const egt_proposal* p);
int proposal_device(const egt_proposal* p);
egt_status run_mesh_1ring(egt_handle* h, int k);
egt_status run_egt(egt_handle* h, float alpha);
egt_status ensure_csr(egt_handle* h);
egt_status csr_nnz(egt_handle* h, int64_t* out);
egt_status run_taubin(egt_handle* h, int iters, float lambda, float mu);
egt_status taubin_launch(const float4* pin, float4* pout, const int* off, const int* col, int n, float scale,
                         cudaStream_t st);
egt_status run_normals(egt_handle* h);
egt_status run_orient(egt_handle* h);
egt_status run_orient_kruskal(const int* knn, float* nrm, int n, int k, int k_use, cudaStream_t st);
egt_status run_output(egt_handle* h, float* x, float* y, float* z);  // device outputs
egt_status lists_original(egt_handle* h, int* out_dev);
egt_status scatter_original(egt_handle* h, const float* soa_sorted, float* soa_orig);
float elapsed_ms(cudaEvent_t a, cudaEvent_t b);
egt_status new_bare_handle(const egt_config& cfg, int64_t n, cudaStream_t stream, egt_handle** out);
void delete_handle(egt_handle* h);
}  // namespace egt
