// C ABI of libegt_b200 (declared in include/egt_b200.h): handle lifecycle,
// argument checking, error reporting and the stage entry points.
#include <cstring>
#include <mutex>
#include <string>
#include "egt_internal.cuh"

namespace egt {

static thread_local std::string g_error;
static thread_local int64_t g_launches = 0;

void count_launch() { g_launches++; }

void set_error(const std::string& msg) { g_error = msg; }

std::string cuda_msg(cudaError_t e, const char* what, const char* file, int line) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s failed: %s (%s) at %s:%d", what, cudaGetErrorName(e),
                  cudaGetErrorString(e), file, line);
    return std::string(buf);
}

float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();
        return -1.f;
    }
    return ms;
}

}  // namespace egt

using namespace egt;

namespace {

egt_status check_handle(egt_handle* h) {
    if (!h) { set_error("null handle"); return EGT_ERR_ARG; }
    return EGT_OK;
}

void bind_stream(egt_handle* h, void* stream) { h->stream = (cudaStream_t)stream; }

void free_handle(egt_handle* h) {
    if (!h) return;
    cudaSetDevice(h->cfg.device);
    auto F = [h](void* p) { dev_free(h, p); };
    F(h->p4); F(h->p4b); F(h->x); F(h->y); F(h->z); F(h->cell0); F(h->perm); F(h->d_norm);
    for (int L = 0; L < kMaxLevels; L++) {
        F(h->lv[L].order); F(h->lv[L].cell_start); F(h->lv[L].cell_x); F(h->lv[L].row_range);
    }
    F(h->lists); F(h->kth); F(h->qlevel); F(h->pclass); F(h->csr_off); F(h->csr_col); F(h->tris); F(h->nrm);
    F(h->d_counters); F(h->scratch.ptr);
    if (h->taubin_exec) cudaGraphExecDestroy(h->taubin_exec);
    F(h->m_perm); F(h->m_inv); F(h->m_p); F(h->m_pb); F(h->m_off); F(h->m_col);
    F(h->t_uni); F(h->t_loc); F(h->t_nu); F(h->t_soff); F(h->tile_mem);
    cudaStreamSynchronize(h->stream);
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    delete h;
}

// Keeps freed pool memory cached in the device's default memory pool.
egt_status warm_pool(int device) {
    static std::mutex mu;
    static bool done[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0 || device >= 64 || done[device]) return EGT_OK;
    cudaMemPool_t pool;
    EGT_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t threshold = ~0ull;
    EGT_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    done[device] = true;
    return EGT_OK;
}

}  // namespace

// A handle with the per-point buffers of n points and no grid (used by the
// batch, which builds its own per-cloud grids).
egt_status egt::new_bare_handle(const egt_config& cfg, int64_t n, cudaStream_t stream, egt_handle** out) {
    *out = nullptr;
    EGT_CUDA_TRY(cudaSetDevice(cfg.device));
    EGT_TRY(::warm_pool(cfg.device));
    egt_handle* h = new egt_handle();
    h->cfg = cfg;
    h->n = n;
    h->stream = stream;
    cudaError_t e = dev_alloc(h, &h->p4, sizeof(float4) * n);
    if (e == cudaSuccess) e = dev_alloc(h, &h->x, sizeof(float) * n);
    if (e == cudaSuccess) e = dev_alloc(h, &h->y, sizeof(float) * n);
    if (e == cudaSuccess) e = dev_alloc(h, &h->z, sizeof(float) * n);
    if (e == cudaSuccess) e = dev_alloc(h, &h->cell0, sizeof(uint32_t) * n);
    if (e == cudaSuccess) e = dev_alloc(h, &h->perm, sizeof(int) * n);
    if (e == cudaSuccess) e = dev_alloc(h, &h->d_counters, sizeof(unsigned long long) * kCtrWords);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->d_counters, 0, sizeof(unsigned long long) * kCtrWords, h->stream);
    for (auto& ev : h->ev)
        if (e == cudaSuccess) e = cudaEventCreate(&ev);
    if (e != cudaSuccess) {
        set_error(cuda_msg(e, "new_bare_handle", __FILE__, __LINE__));
        free_handle(h);
        return e == cudaErrorMemoryAllocation ? EGT_ERR_NOMEM : EGT_ERR_CUDA;
    }
    *out = h;
    return EGT_OK;
}

void egt::delete_handle(egt_handle* h) { free_handle(h); }

namespace {

egt_status create_common(const float* xyz, bool xyz_on_device, int64_t n, const uint32_t* tris, int64_t t,
                         const egt_config* cfg_in, void* stream, egt_handle** out) {
    if (!out) { set_error("null output handle pointer"); return EGT_ERR_ARG; }
    *out = nullptr;
    if (!xyz) { set_error("null point array"); return EGT_ERR_ARG; }
    if (n < 1 || n > (int64_t)(1u << 30)) { set_error("point count must be in [1, 2^30]"); return EGT_ERR_ARG; }
    if (t < 0 || (t > 0 && !tris)) { set_error("invalid triangle array"); return EGT_ERR_ARG; }
    egt_config cfg;
    egt_default_config(&cfg);
    if (cfg_in) cfg = *cfg_in;
    if (cfg.bucket_count != 1024) {
        set_error("bucket_count must be 1024 (the reference's level-0 grid)");
        return EGT_ERR_ARG;
    }
    if (cfg.max_points_in_cell < 1) { set_error("max_points_in_cell must be >= 1"); return EGT_ERR_ARG; }
    if (cfg.knn_mode != EGT_KNN_PLAIN && cfg.knn_mode != EGT_KNN_LEARNED && cfg.knn_mode != EGT_KNN_SELECT &&
        cfg.knn_mode != EGT_KNN_TILE) {
        set_error("knn_mode must be EGT_KNN_PLAIN, EGT_KNN_LEARNED, EGT_KNN_SELECT or EGT_KNN_TILE");
        return EGT_ERR_ARG;
    }
    EGT_CUDA_TRY(cudaSetDevice(cfg.device));
    EGT_TRY(warm_pool(cfg.device));
    egt_handle* h = new egt_handle();
    h->cfg = cfg;
    h->n = n;
    h->is_mesh = tris != nullptr;
    h->t = t;
    bind_stream(h, stream);
    auto fail = [&](egt_status s) { free_handle(h); return s; };
#define CREATE_TRY(call)                                                     \
    do {                                                                     \
        cudaError_t e__ = (call);                                            \
        if (e__ != cudaSuccess) {                                            \
            set_error(cuda_msg(e__, #call, __FILE__, __LINE__));             \
            return fail(e__ == cudaErrorMemoryAllocation ? EGT_ERR_NOMEM : EGT_ERR_CUDA); \
        }                                                                    \
    } while (0)
    CREATE_TRY(dev_alloc(h, &h->p4, sizeof(float4) * n));
    CREATE_TRY(dev_alloc(h, &h->x, sizeof(float) * n));
    CREATE_TRY(dev_alloc(h, &h->y, sizeof(float) * n));
    CREATE_TRY(dev_alloc(h, &h->z, sizeof(float) * n));
    CREATE_TRY(dev_alloc(h, &h->cell0, sizeof(uint32_t) * n));
    CREATE_TRY(dev_alloc(h, &h->perm, sizeof(int) * n));
    CREATE_TRY(dev_alloc(h, &h->d_norm, sizeof(NormParams)));
    CREATE_TRY(dev_alloc(h, &h->d_counters, sizeof(unsigned long long) * kCtrWords));
    CREATE_TRY(cudaMemsetAsync(h->d_counters, 0, sizeof(unsigned long long) * kCtrWords, h->stream));
    for (auto& e : h->ev) CREATE_TRY(cudaEventCreate(&e));
    const float* dxyz = xyz;
    float* staged = nullptr;
    if (!xyz_on_device) {
        CREATE_TRY(cudaMallocAsync((void**)&staged, sizeof(float) * 3 * n, h->stream));
        CREATE_TRY(cudaMemcpyAsync(staged, xyz, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, h->stream));
        dxyz = staged;
    }
    if (tris && t > 0) {
        CREATE_TRY(dev_alloc(h, &h->tris, sizeof(uint32_t) * 3 * t));
        CREATE_TRY(cudaMemcpyAsync(h->tris, tris, sizeof(uint32_t) * 3 * t, cudaMemcpyHostToDevice, h->stream));
    }
    egt_status s = build_grid(h, dxyz, h->is_mesh ? 1 : kMaxLevels);
    if (staged) cudaFreeAsync(staged, h->stream);
    if (s != EGT_OK) return fail(s);
    CREATE_TRY(cudaStreamSynchronize(h->stream));
#undef CREATE_TRY
    h->tm.grid_ms = elapsed_ms(h->ev[0], h->ev[1]);
    *out = h;
    return EGT_OK;
}

}  // namespace

extern "C" {

void egt_default_config(egt_config* cfg) {
    if (!cfg) return;
    cfg->device = 0;
    cfg->eps = 1e-6f;
    cfg->bucket_count = 1024;
    cfg->threshold = 1e8f;
    cfg->max_points_in_cell = 100000;
    cfg->knn_mode = EGT_KNN_TILE;
    cfg->warps_per_block = 0;
    cfg->normals_gap_tol = 0.1f;
}

const char* egt_last_error(void) { return g_error.c_str(); }

const char* egt_version(void) { return "egt_b200 1.0 (sm_100a)"; }

egt_status egt_create_cloud(const float* xyz_host, int64_t n, const egt_config* cfg, void* stream,
                            egt_handle** out) {
    return create_common(xyz_host, false, n, nullptr, 0, cfg, stream, out);
}

egt_status egt_create_cloud_device(const float* xyz_dev, int64_t n, const egt_config* cfg, void* stream,
                                   egt_handle** out) {
    return create_common(xyz_dev, true, n, nullptr, 0, cfg, stream, out);
}

egt_status egt_create_mesh(const float* xyz_host, int64_t n, const uint32_t* tris_host, int64_t t,
                           const egt_config* cfg, void* stream, egt_handle** out) {
    if (!tris_host || t < 1) { set_error("a mesh needs at least one triangle"); return EGT_ERR_ARG; }
    return create_common(xyz_host, false, n, tris_host, t, cfg, stream, out);
}

egt_status egt_update_points_device(egt_handle* h, const float* xyz_dev, void* stream) {
    EGT_TRY(check_handle(h));
    if (!xyz_dev) { set_error("egt_update_points_device: null points"); return EGT_ERR_ARG; }
    if (h->is_mesh) { set_error("egt_update_points_device: point-cloud handles only"); return EGT_ERR_STATE; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    h->have_csr = false;
    if (h->nrm) { dev_free(h, h->nrm); h->nrm = nullptr; }
    return build_grid(h, xyz_dev, kMaxLevels);
}

int64_t egt_kernel_launches(void) { return g_launches; }

egt_status egt_set_threshold(egt_handle* h, float thres, void* stream) {
    EGT_TRY(check_handle(h));
    if (!(thres > 0.0f)) { set_error("egt_set_threshold: thres must be > 0"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    return set_threshold(h, thres);
}

egt_status egt_knn(egt_handle* h, int k, void* stream) {
    EGT_TRY(check_handle(h));
    if (h->is_mesh) { set_error("egt_knn: mesh handles take their neighbours from triangles"); return EGT_ERR_STATE; }
    if ((int64_t)k * h->n > (int64_t)0x7fffffff) { set_error("egt_knn: n*k exceeds 2^31-1"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    if (h->cfg.knn_mode == EGT_KNN_LEARNED) {
        if (!h->proposal) { set_error("egt_knn: learned mode needs egt_attach_proposal"); return EGT_ERR_STATE; }
        return egt_knn_learned(h, k, h->proposal, stream);
    }
    h->last_knn_learned = false;
    return run_knn(h, k);
}

egt_status egt_knn_host(egt_handle* h, int k, int* knn_host, void* stream) {
    EGT_TRY(check_handle(h));
    if (!knn_host) { set_error("egt_knn_host: null output"); return EGT_ERR_ARG; }
    if (h->is_mesh) { set_error("egt_knn_host: mesh handles take their neighbours from triangles"); return EGT_ERR_STATE; }
    if ((int64_t)k * h->n > (int64_t)0x7fffffff) { set_error("egt_knn_host: n*k exceeds 2^31-1"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    // The chunked ring search overlaps each chunk's copy with the next chunk's
    // search.  The cell-tile search completes cell by cell, not in row order,
    // so its copy could only follow the whole search: measured slower end to
    // end (4M points, k = 40: 33.6 ms against 27.2 ms), so EGT_KNN_TILE uses
    // the chunked ring search here.
    if (h->cfg.knn_mode == EGT_KNN_LEARNED) {  // no chunked form: search, then copy
        EGT_TRY(egt_knn(h, k, stream));
        return egt_get_knn_host(h, knn_host, stream);
    }
    h->last_knn_learned = false;
    return run_knn_host(h, k, knn_host);
}

egt_status egt_knn_query(egt_handle* h, const float* queries_host, int64_t nq, int k, int* knn_host,
                         int64_t* invalid, void* stream) {
    EGT_TRY(check_handle(h));
    if (h->is_mesh) { set_error("egt_knn_query: point-cloud handles only"); return EGT_ERR_STATE; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    return run_knn_query(h, queries_host, nq, k, knn_host, invalid);
}

egt_status egt_orient_kruskal(const int* knn, float* nx, float* ny, float* nz, const float* x, const float* y,
                              const float* z, int n, int k, int k_use, int device, void* stream) {
    (void)x; (void)y; (void)z;  // in the reference's signature, not read by it either
    if (n < 0 || k < 1 || k_use < 0 || k_use > k) {
        set_error("egt_orient_kruskal: need n >= 0, k >= 1 and 0 <= k_use <= k");
        return EGT_ERR_ARG;
    }
    if (n == 0 || k_use == 0) return EGT_OK;
    if (!knn || !nx || !ny || !nz) { set_error("egt_orient_kruskal: null array"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(device));
    cudaStream_t st = (cudaStream_t)stream;
    int* d_knn = nullptr;
    float* d_nrm = nullptr;
    // whole rows: one contiguous copy (a strided copy of k_use columns from
    // pageable memory goes row by row)
    EGT_CUDA_TRY(cudaMallocAsync((void**)&d_knn, sizeof(int) * (size_t)n * k, st));
    EGT_CUDA_TRY(cudaMallocAsync((void**)&d_nrm, sizeof(float) * 3 * (size_t)n, st));
    egt_status s = EGT_OK;
    cudaError_t e = cudaMemcpyAsync(d_knn, knn, sizeof(int) * (size_t)n * k, cudaMemcpyHostToDevice, st);
    const float* src[3] = {nx, ny, nz};
    for (int c = 0; c < 3 && e == cudaSuccess; c++)
        e = cudaMemcpyAsync(d_nrm + (size_t)c * n, src[c], sizeof(float) * n, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) { set_error(cuda_msg(e, "egt_orient_kruskal upload", __FILE__, __LINE__)); s = EGT_ERR_CUDA; }
    if (s == EGT_OK) s = run_orient_kruskal(d_knn, d_nrm, n, k, k_use, st);
    if (s == EGT_OK) {
        float* dst[3] = {nx, ny, nz};
        for (int c = 0; c < 3 && e == cudaSuccess; c++)
            e = cudaMemcpyAsync(dst[c], d_nrm + (size_t)c * n, sizeof(float) * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { set_error(cuda_msg(e, "egt_orient_kruskal download", __FILE__, __LINE__)); s = EGT_ERR_CUDA; }
    }
    cudaFreeAsync(d_knn, st);
    cudaFreeAsync(d_nrm, st);
    cudaStreamSynchronize(st);
    return s;
}

egt_status egt_knn_learned(egt_handle* h, int k, const egt_proposal* p, void* stream) {
    EGT_TRY(check_handle(h));
    if (!p) { set_error("egt_knn_learned: null proposal"); return EGT_ERR_ARG; }
    if (h->is_mesh) { set_error("egt_knn_learned: point-cloud handles only"); return EGT_ERR_STATE; }
    if ((int64_t)k * h->n > (int64_t)0x7fffffff) { set_error("egt_knn_learned: n*k exceeds 2^31-1"); return EGT_ERR_ARG; }
    if (proposal_k(p) != k) { set_error("egt_knn_learned: k differs from the proposal's k"); return EGT_ERR_ARG; }
    if (proposal_device(p) != h->cfg.device) { set_error("egt_knn_learned: proposal on another device"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    h->last_knn_learned = true;
    return run_knn_learned(h, k, p);
}

egt_status egt_attach_proposal(egt_handle* h, const egt_proposal* p) {
    EGT_TRY(check_handle(h));
    if (p && proposal_device(p) != h->cfg.device) { set_error("egt_attach_proposal: proposal on another device"); return EGT_ERR_ARG; }
    h->proposal = p;
    return EGT_OK;
}

egt_status egt_mesh_1ring(egt_handle* h, int k, void* stream) {
    EGT_TRY(check_handle(h));
    if ((int64_t)k * h->n > (int64_t)0x7fffffff) { set_error("egt_mesh_1ring: n*k exceeds 2^31-1"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    return run_mesh_1ring(h, k);
}

egt_status egt_filter(egt_handle* h, float alpha, void* stream) {
    EGT_TRY(check_handle(h));
    if (!(alpha > 0.f)) { set_error("egt_filter: alpha must be > 0"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    return run_egt(h, alpha);
}

egt_status egt_taubin(egt_handle* h, int iters, float lambda, float mu, void* stream) {
    EGT_TRY(check_handle(h));
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    return run_taubin(h, iters, lambda, mu);
}

egt_status egt_smooth(egt_handle* h, int iters, float lambda, float mu, float alpha, void* stream) {
    EGT_TRY(egt_filter(h, alpha, stream));
    return egt_taubin(h, iters, lambda, mu, stream);
}

egt_status egt_normals(egt_handle* h, float* nx, float* ny, float* nz, void* stream) {
    EGT_TRY(check_handle(h));
    if (h->is_mesh) { set_error("egt_normals: normals are computed for point clouds only"); return EGT_ERR_STATE; }
    if (!h->lists) { set_error("egt_normals: no neighbour lists"); return EGT_ERR_STATE; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    EGT_TRY(run_normals(h));
    EGT_TRY(run_orient(h));
    if (nx || ny || nz) {
        if (!nx || !ny || !nz) { set_error("egt_normals: give all three outputs or none"); return EGT_ERR_ARG; }
        const int64_t n = h->n;
        float* tmp = nullptr;
        EGT_CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(float) * 3 * n, h->stream));
        // scatter sorted-space normals to original order (rearrange_output, Normal_CUDA.cu:745-759)
        EGT_TRY(scatter_original(h, h->nrm, tmp));
        EGT_CUDA_TRY(cudaMemcpyAsync(nx, tmp, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
        EGT_CUDA_TRY(cudaMemcpyAsync(ny, tmp + n, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
        EGT_CUDA_TRY(cudaMemcpyAsync(nz, tmp + 2 * n, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
        cudaFreeAsync(tmp, h->stream);
        EGT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
    return EGT_OK;
}

egt_status egt_output_device(egt_handle* h, float* x, float* y, float* z, void* stream) {
    EGT_TRY(check_handle(h));
    if (!x || !y || !z) { set_error("egt_output: null output"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    return run_output(h, x, y, z);
}

egt_status egt_output(egt_handle* h, float* x, float* y, float* z, void* stream) {
    EGT_TRY(check_handle(h));
    if (!x || !y || !z) { set_error("egt_output: null output"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    const int64_t n = h->n;
    float* tmp = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(float) * 3 * n, h->stream));
    egt_status s = run_output(h, tmp, tmp + n, tmp + 2 * n);
    if (s == EGT_OK) {
        EGT_CUDA_TRY(cudaMemcpyAsync(x, tmp, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
        EGT_CUDA_TRY(cudaMemcpyAsync(y, tmp + n, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
        EGT_CUDA_TRY(cudaMemcpyAsync(z, tmp + 2 * n, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
    }
    cudaFreeAsync(tmp, h->stream);
    EGT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return s;
}

egt_status egt_get_knn_host(egt_handle* h, int* knn_host, void* stream) {
    EGT_TRY(check_handle(h));
    if (!knn_host) { set_error("egt_get_knn_host: null output"); return EGT_ERR_ARG; }
    if (!h->lists) { set_error("egt_get_knn_host: no neighbour lists"); return EGT_ERR_STATE; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    const size_t tot = (size_t)h->n * h->k;
    int* tmp = nullptr;
    EGT_CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(int) * tot, h->stream));
    egt_status s = lists_original(h, tmp);
    if (s == EGT_OK)
        EGT_CUDA_TRY(cudaMemcpyAsync(knn_host, tmp, sizeof(int) * tot, cudaMemcpyDeviceToHost, h->stream));
    cudaFreeAsync(tmp, h->stream);
    EGT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return s;
}

}  // extern "C"

namespace {
// Positions a KNNInterface consumer left in the provider's slots (device SoA,
// sorted space) into the handle's float4 array; the slot arrays are copied
// into the handle's SoA mirror when they are not that mirror.
__global__ void k_commit_positions(const float* __restrict__ x, const float* __restrict__ y,
                                   const float* __restrict__ z, int64_t n, float4* __restrict__ p4, float* hx,
                                   float* hy, float* hz) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float vx = x[i], vy = y[i], vz = z[i];
    float4 p = p4[i];
    p.x = vx; p.y = vy; p.z = vz;
    p4[i] = p;
    if (x != hx) hx[i] = vx;
    if (y != hy) hy[i] = vy;
    if (z != hz) hz[i] = vz;
}
}  // namespace

extern "C" {

egt_status egt_taubin_halfstep(const float* pos_in, float* pos_out, const int* csr_off, const int* csr_col,
                               int64_t rows, float scale, int device, void* stream) {
    if (rows < 0 || rows > (int64_t)0x7fffffff) { set_error("egt_taubin_halfstep: rows out of range"); return EGT_ERR_ARG; }
    if (rows == 0) return EGT_OK;
    if (!pos_in || !pos_out || !csr_off || !csr_col) {
        set_error("egt_taubin_halfstep: null pointer argument");
        return EGT_ERR_ARG;
    }
    if (pos_in == pos_out) { set_error("egt_taubin_halfstep: pos_in and pos_out must not alias"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(device));
    return taubin_launch(reinterpret_cast<const float4*>(pos_in), reinterpret_cast<float4*>(pos_out), csr_off,
                         csr_col, (int)rows, scale, (cudaStream_t)stream);
}

egt_status egt_commit_views(egt_handle* h, const float* x, const float* y, const float* z, void* stream) {
    EGT_TRY(check_handle(h));
    if (!x || !y || !z) { set_error("egt_commit_views: null position array"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    bind_stream(h, stream);
    const unsigned T = 256;
    k_commit_positions<<<(unsigned)((h->n + T - 1) / T), T, 0, h->stream>>>(x, y, z, h->n, h->p4, h->x, h->y,
                                                                             h->z);
    EGT_LAUNCH_CHECK();
    // the lists may have been rewritten in place: neighbourhoods are rebuilt
    // from them by the next stage that needs them
    h->have_csr = false;
    return EGT_OK;
}

egt_status egt_free_device(void* p) {
    if (p) EGT_CUDA_TRY(cudaFree(p));
    return EGT_OK;
}

egt_status egt_get_views(egt_handle* h, egt_views* v) {
    EGT_TRY(check_handle(h));
    if (!v) { set_error("egt_get_views: null output"); return EGT_ERR_ARG; }
    v->x = h->x;
    v->y = h->y;
    v->z = h->z;
    v->lists = h->lists;
    v->perm = h->perm;
    v->normals = h->nrm;
    v->n = h->n;
    v->k = h->k;
    v->min_extent = h->norm.mn;
    v->max_extent = h->norm.mx;
    return EGT_OK;
}

egt_status egt_get_csr(egt_handle* h, const int** offsets, const int** cols, int64_t* nnz) {
    EGT_TRY(check_handle(h));
    if (!h->lists) { set_error("egt_get_csr: no neighbour lists"); return EGT_ERR_STATE; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    EGT_TRY(ensure_csr(h));
    int64_t m = 0;
    EGT_TRY(csr_nnz(h, &m));
    if (offsets) *offsets = h->csr_off;
    if (cols) *cols = h->csr_col;
    if (nnz) *nnz = m;
    return EGT_OK;
}

egt_status egt_get_timings(egt_handle* h, egt_timings* t) {
    EGT_TRY(check_handle(h));
    if (!t) { set_error("egt_get_timings: null output"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    EGT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    unsigned long long ctr[kCtrWords];
    EGT_CUDA_TRY(cudaMemcpy(ctr, h->d_counters, sizeof(ctr), cudaMemcpyDeviceToHost));
    h->tm.knn_ms = elapsed_ms(h->ev[2], h->ev[3]);
    h->tm.egt_ms = elapsed_ms(h->ev[4], h->ev[5]);
    h->tm.egt_kernel_ms = elapsed_ms(h->ev[4], h->ev[14]);
    h->tm.taubin_ms = elapsed_ms(h->ev[6], h->ev[7]);
    h->tm.normals_ms = elapsed_ms(h->ev[8], h->ev[9]);
    h->tm.orient_ms = elapsed_ms(h->ev[10], h->ev[11]);
    h->tm.output_ms = elapsed_ms(h->ev[12], h->ev[13]);
    h->tm.invalid_queries = (int64_t)ctr[kCtrInvalid];
    h->tm.levels_used = (int)ctr[kCtrMaxLevel];
    if (h->have_csr) EGT_TRY(csr_nnz(h, &h->tm.csr_nnz));
    h->tm.normals_fp64 = (int64_t)ctr[kCtrNormFallback];
    h->tm.msf_edges = (int64_t)ctr[kCtrMsf];
    h->tm.components = (int)ctr[kCtrComps];
    h->tm.exact_reruns = (int64_t)ctr[kCtrExactRerun];
    h->tm.knn_fallback = h->last_knn_learned ? 0 : (int64_t)(ctr[kCtrSelFallback] + ctr[kCtrTileRing2]);
    h->tm.knn_evaluations = h->last_knn_learned ? 0 : (int64_t)ctr[kCtrEvals];
    h->tm.egt_tests = (int64_t)ctr[kCtrEgtTests];
    h->tm.taubin_spill_tiles = h->tm.taubin_tiles > 0 ? (int64_t)ctr[kCtrSpillTiles] : 0;
    if (h->last_knn_learned) {
        h->tm.propose_ms = elapsed_ms(h->ev[2], h->ev[15]);
        h->tm.box_queries = (int64_t)ctr[kCtrBoxTried];
        h->tm.certified_queries = (int64_t)ctr[kCtrCertified];
    } else {
        h->tm.propose_ms = 0.0f;
        h->tm.box_queries = 0;
        h->tm.certified_queries = 0;
    }
    *t = h->tm;
    return EGT_OK;
}

egt_status egt_copy_to_host(egt_handle* h, void* dst, const void* src, int64_t bytes) {
    EGT_TRY(check_handle(h));
    if (bytes < 0 || (bytes > 0 && (!dst || !src))) { set_error("egt_copy_to_host: bad arguments"); return EGT_ERR_ARG; }
    EGT_CUDA_TRY(cudaSetDevice(h->cfg.device));
    EGT_CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (bytes) EGT_CUDA_TRY(cudaMemcpy(dst, src, (size_t)bytes, cudaMemcpyDeviceToHost));
    return EGT_OK;
}

void egt_destroy(egt_handle* h) {
    if (!h) return;
    cudaSetDevice(h->cfg.device);
    cudaStreamSynchronize(h->stream);
    free_handle(h);
}

}  // extern "C"
