/*
 * egt_b200.h -- C ABI of the B200-native grid kNN / elliptic-Gabriel / Taubin /
 * normals path.  Plain pointers and sizes only; every call returns an
 * egt_status (0 = success, negative = error) and takes an explicit CUDA stream
 * (cudaStream_t passed as void*, NULL = legacy default stream).
 *
 * The reference (agalex1974/MultiGPUEGTSmoothing) has no C ABI; its drop-in
 * boundary is the C++ provider class KNNInterface (KNNInterface.cuh:8-31) and
 * the classes that produce and consume it.  Each entry point below names the
 * reference interface it replaces.  A handle owns every device buffer, like the
 * reference providers do (GridKNNCuda.cu:1005-1021).  Handles are not
 * thread-safe; separate handles on separate streams are independent.
 *
 * Index spaces: "sorted" = cell-sorted order produced at creation (the order
 * of the reference's device arrays, GridKNNCuda.cu:1114-1128); "original" =
 * input order.  Device positions are normalised into the unit cube with one
 * scalar extent for all axes (GridKNNCuda.cu:1042-1071).
 */
#ifndef EGT_B200_H
#define EGT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int egt_status;
#define EGT_OK                 0
#define EGT_ERR_CUDA          -1  /* a CUDA runtime call failed (see egt_last_error) */
#define EGT_ERR_ARG           -2  /* invalid argument (null pointer, n/k out of range) */
#define EGT_ERR_CAP_EXCEEDED  -3  /* a bounded loop or buffer cap was exceeded */
#define EGT_ERR_TIMEOUT       -4  /* a bounded device wait expired */
#define EGT_ERR_STATE         -5  /* call out of order (e.g. smoothing before kNN) */
#define EGT_ERR_NOMEM         -6  /* device allocation failed */

typedef struct egt_handle egt_handle;
typedef struct egt_proposal egt_proposal;

/* Learned search proposal network (no reference counterpart): 8 features ->
 * 32 -> 32 -> 16 classes, binary16 parameters. */
#define EGT_PROPOSAL_FEATURES 8
#define EGT_PROPOSAL_CLASSES 16
#define EGT_PROPOSAL_PARAMS 1872

#define EGT_KNN_PLAIN 0    /* the reference's ring expansion, one warp per query */
#define EGT_KNN_LEARNED 1  /* proposal-driven box search, certified rows; the ring search for the rest */
#define EGT_KNN_SELECT 2   /* block selection, certified rows; the ring search for the rest */
#define EGT_KNN_TILE 3     /* cell tiles (default): a cell's queries one per lane over its 3x3x3
                              block, certified rows; the ring search for the rest.  For 16 <= k <= 64;
                              other k use the ring search */

/* Tunables.  Defaults reproduce the reference CLI (main.cpp:108-116). */
typedef struct egt_config {
    int device;              /* CUDA device ordinal (default 0) */
    float eps;               /* cube widening, GridStructure eps (1e-6) */
    int bucket_count;        /* level-0 buckets per axis (1024) */
    float threshold;         /* GRIDCUDAKNNSELF_COMPACT thres before scaling (1e8) */
    int max_points_in_cell;  /* MAX_PNTS_IN_CUBE (100000): larger cells invalidate a query */
    int knn_mode;            /* EGT_KNN_TILE (default), EGT_KNN_PLAIN, EGT_KNN_SELECT, or
                                EGT_KNN_LEARNED: egt_knn uses the proposal attached with
                                egt_attach_proposal.  All four give identical lists. */
    int warps_per_block;     /* kNN/EGT launch shape (0 = autotuned default) */
    float normals_gap_tol;   /* FP64 eigensolve when (l1-l0) < tol*l2 (0.1; 0 = FP32 only) */
} egt_config;

/* Device views for the KNNInterface adapter (include/egt_knn_interface.hpp). */
typedef struct egt_views {
    float* x;                /* [n] sorted, normalised (GetRefPointsX()[0]) */
    float* y;                /* [n] (GetRefPointsY()[0]) */
    float* z;                /* [n] (GetRefPointsZ()[0]) */
    int* lists;              /* [n*k] sorted-space lists, -1 padded (GetKNNIndexesInPartitions()[0]) */
    int* perm;               /* [n] sorted slot -> original index (GetOriginalRefIndexes()[0]) */
    float* normals;          /* [3n] SoA sorted-space normals after egt_normals, else NULL */
    int64_t n;               /* pointsRefCount() */
    int k;                   /* NeighborCount() (0 before a neighbour search) */
    float min_extent;        /* GetMinExtent() */
    float max_extent;        /* GetMaxExtent() */
} egt_views;

/* Per-stage device times of the last calls on a handle, in milliseconds. */
typedef struct egt_timings {
    float grid_ms, knn_ms, egt_ms, taubin_ms, normals_ms, orient_ms, output_ms;
    int levels_used;         /* deepest hierarchy level any query reached (0..7) */
    int64_t invalid_queries; /* rows set to -1 by the invalidation rules */
    int64_t csr_nnz;         /* neighbours kept by the EGT filter */
    int64_t normals_fp64;    /* points whose normal was re-solved in FP64 */
    int64_t msf_edges;       /* edges of the orientation spanning forest */
    int components;          /* orientation components (trees with >= 1 edge) */
    float egt_kernel_ms;     /* the EGT filter kernel alone (egt_ms also packs the CSR) */
    float propose_ms;        /* learned kNN: features + proposal network (inside knn_ms) */
    int64_t box_queries;     /* learned kNN: queries that ran a proposed box search */
    int64_t certified_queries; /* learned kNN: box results certified (the rest ran the plain search) */
    int64_t exact_reruns;    /* kNN queries whose kept distances tied and that were searched again
                                with the reference's one-at-a-time insertion rule */
    int64_t knn_evaluations; /* kNN: candidate distances evaluated (8 FP32 operations each; the cell-tile
                                search counts each candidate once per query though it computes it twice) */
    int64_t egt_tests;       /* EGT filter: ellipsoid tests evaluated (24 FP32 operations each) */
    int64_t taubin_tiles;    /* 256-row tiles of the staged Taubin half-step (last CSR smoothed) */
    int64_t taubin_spill_tiles; /* of those, tiles too large to stage in shared memory, whose rows
                                   gather their neighbours from global memory */
    int64_t knn_fallback;    /* EGT_KNN_SELECT / EGT_KNN_TILE: queries the block selection or the cell
                                tiles did not certify (equal distances, oversized cells, a k-th ball
                                beyond the block, ...) or did not take, which the ring search ran */
} egt_timings;

void egt_default_config(egt_config* cfg);
const char* egt_last_error(void);
const char* egt_version(void);

/* GridStructure(mesh, 1, eps, 1024, 4) (GridKNNCuda.cu:1165-1205 + InitStructure
 * :1023-1133): copies n points (AoS xyz, host memory), normalises them, sorts
 * them by cell and builds the cell hierarchy. */
egt_status egt_create_cloud(const float* xyz_host, int64_t n, const egt_config* cfg, void* stream,
                            egt_handle** out);
/* Same, with the points already in device memory (AoS xyz). */
egt_status egt_create_cloud_device(const float* xyz_dev, int64_t n, const egt_config* cfg, void* stream,
                                   egt_handle** out);
/* GridMeshCuda(mesh, 1, eps, 1024) (GridMeshCuda1.cu:247-414): points plus
 * t triangles (uint32 vertex indices, host memory). */
egt_status egt_create_mesh(const float* xyz_host, int64_t n, const uint32_t* tris_host, int64_t t,
                           const egt_config* cfg, void* stream, egt_handle** out);

/* Re-runs InitStructure for new positions of the same n points (device AoS
 * xyz), reusing every buffer of the handle: normalisation, cell sort and
 * hierarchy are rebuilt, previous lists/CSR/normals are invalidated. */
egt_status egt_update_points_device(egt_handle* h, const float* xyz_dev, void* stream);

/* GridStructure::GRIDCUDAKNNSELF_COMPACT(k, thres) (GridKNNCuda.cu:2322-2634),
 * with the handle's threshold (egt_config.threshold, or egt_set_threshold). */
egt_status egt_knn(egt_handle* h, int k, void* stream);
/* The thres argument of GRIDCUDAKNNSELF_COMPACT / GRIDCUDAKNNCompact
 * (GridKNNCuda.cu:2324-2325, :1667-1668): the admission threshold of the
 * following searches on h, in the reference's units (scaled by the
 * normalisation extent and squared on the device).  thres > 0. */
egt_status egt_set_threshold(egt_handle* h, float thres, void* stream);
/* GridMeshCuda::GetNeighborsFromTriangles(k) (GridMeshCuda1.cu:416-511). */
egt_status egt_mesh_1ring(egt_handle* h, int k, void* stream);

/* EGT_CUDA::PerformSmoothing(iters, lambda, mu, alpha) (EGT_CUDA.cu:476-648):
 * the elliptic-Gabriel filter followed by iters lambda/mu Taubin iterations. */
egt_status egt_smooth(egt_handle* h, int iters, float lambda, float mu, float alpha, void* stream);
/* The two halves of egt_smooth: calculateEGG_GKNN (EGT_CUDA.cu:172-189, :505-530)
 * and the Taubin loop (EGT_CUDA.cu:229-276, :559-633). */
egt_status egt_filter(egt_handle* h, float alpha, void* stream);
egt_status egt_taubin(egt_handle* h, int iters, float lambda, float mu, void* stream);

/* Normal_CUDA::GetNormals(nx, ny, nz) (Normal_CUDA.cu:304-775): oriented
 * normals in original order, written to host (or NULL to keep them on device). */
egt_status egt_normals(egt_handle* h, float* nx, float* ny, float* nz, void* stream);

/* getOutputPoints(x, y, z, provider) (getOutputPoints.cu:34-63): denormalised
 * positions in original order, written to host memory. */
egt_status egt_output(egt_handle* h, float* x, float* y, float* z, void* stream);
/* Same, written to device memory (SoA, original order). */
egt_status egt_output_device(egt_handle* h, float* x, float* y, float* z, void* stream);

/* KNNInterface::GetKNNIndexes (GridKNNCuda.cu:1941-1968): n*k host ints in
 * original ids and original row order. */
egt_status egt_get_knn_host(egt_handle* h, int* knn_host, void* stream);
/* egt_knn followed by egt_get_knn_host -- GRIDCUDAKNNSELF_COMPACT(k) then
 * GetKNNIndexes (GridKNNCuda.cu:2322-2634, :1941-1968) -- with the host copy
 * overlapped: the queries are searched in chunks of original rows, and each
 * chunk's rows are copied to knn_host (n*k ints; pinned memory lets the copy
 * overlap) while the next chunk is searched.  The handle's lists are those
 * of egt_knn.  The chunks run the ring search in every mode but
 * EGT_KNN_LEARNED, where the search and the copy run one after the other
 * (the cell-tile search finishes cell by cell, not in row order, so its copy
 * could not start early). */
egt_status egt_knn_host(egt_handle* h, int k, int* knn_host, void* stream);

/* Query-vs-reference kNN against the handle's points:
 * GridStructure::GRIDCUDAKNNCompact(qx, qy, qz, nq, k, thres) then
 * GetKNNIndexes (GridKNNCuda.cu:1645-1968).  queries_host: nq*3 floats (AoS,
 * the reference's units; they may lie outside its cube); knn_host: nq*k ints,
 * original reference ids in query order, -1 padded (an invalid query's row is
 * all -1); invalid (optional): number of invalid queries.  thres is the
 * handle's configured threshold.  The handle's own lists are not changed. */
egt_status egt_knn_query(egt_handle* h, const float* queries_host, int64_t nq, int k, int* knn_host,
                         int64_t* invalid, void* stream);
/* orient_kruskal(knn, nx, ny, nz, x, y, z, N, k, k_use) (MST.cpp:399-423, with
 * Graph::kruskalMST :297-376 and orientSpanningTree :262-279): the
 * reference's CPU normal orienter, computed on the GPU with identical results.
 * Host arrays, as in the reference: knn n*k ints (row i lists the neighbours of
 * point i, entries < 0 are empty; only the first k_use of each row are read;
 * an entry >= n is rejected with EGT_ERR_ARG), nx/ny/nz n floats each,
 * oriented in place.  The edges are the distinct list pairs, weighted
 * max(0, 1 - |n_u . n_v|) and ordered by (weight, u, v); each tree of the
 * minimum spanning forest is walked from its union-find root, negating a
 * normal whose dot product with its parent's is negative.  x, y, z are part
 * of the reference's signature and are not read (they may be NULL).  The
 * reference forms its edge key in 32-bit int arithmetic, which overflows
 * above 46,340 points; this entry point uses 64-bit keys.  device: CUDA
 * device ordinal; stream may be NULL. */
egt_status egt_orient_kruskal(const int* knn, float* nx, float* ny, float* nz, const float* x, const float* y,
                              const float* z, int n, int k, int k_use, int device, void* stream);

/* Device pointers behind the KNNInterface getters. */
egt_status egt_get_views(egt_handle* h, egt_views* views);
/* Hands back what a KNNInterface consumer left in the provider's slots, as the
 * reference's consumers leave it (EGT_CUDA::PerformSmoothing writes smoothed
 * positions through GetRefPointsX/Y/Z()[0] and may swap those pointers,
 * EGT_CUDA.cu:591-632; calculateEGG_GKNN writes -1 into the lists in place,
 * EGT_CUDA.cu:172-189): x, y, z are the arrays now in the slots (device SoA,
 * sorted space, normalised; the handle's own views or a consumer's buffers),
 * copied into the handle; the lists are taken as rewritten, so later stages
 * rebuild their neighbourhoods from them. */
egt_status egt_commit_views(egt_handle* h, const float* x, const float* y, const float* z, void* stream);
/* cudaFree for a device buffer a KNNInterface consumer swapped into a
 * provider slot: the provider frees whatever its slots hold at destruction
 * (GridKNNCuda.cu:1005-1021). */
egt_status egt_free_device(void* p);
/* Per-stage device timings of the last calls (filled when the stream is synced). */
egt_status egt_get_timings(egt_handle* h, egt_timings* t);
/* Sorted-space EGT-filtered neighbourhoods as CSR (device pointers, valid
 * until the next call on the handle): offsets [n+1], cols [nnz]. */
egt_status egt_get_csr(egt_handle* h, const int** offsets, const int** cols, int64_t* nnz);

/* One half-step of taubin_step_GKNN (EGT_CUDA.cu:229-276) over rows
 * [0, rows) of a CSR -- the per-GPU step of the reference's partitioned
 * smoothing (EGT_CUDA.cu:559-633), whose halo exchange the caller does:
 * pos_in: device float4 (x,y,z,w) positions indexed by csr_col (row i's own
 * position is pos_in[i]; entries past the rows hold the halo), pos_out: rows
 * float4 (w copied), not aliasing pos_in; scale: lambda or mu.  Allocates
 * nothing. */
egt_status egt_taubin_halfstep(const float* pos_in, float* pos_out, const int* csr_off, const int* csr_col,
                               int64_t rows, float scale, int device, void* stream);

/* Taubin lambda/mu smoothing that allocates no device memory, for callers that
 * cannot allocate: hosts whose single allocator (a caching allocator or a
 * pre-sized arena) owns all GPU memory, where a cudaMalloc can fail or
 * fragment it, and real-time loops that cannot take the device
 * synchronisation of cudaMalloc/cudaFree.  No counterpart in the reference.
 * pos_in/pos_out: n float4 (x,y,z,w) in device memory (may alias);
 * csr_off [n+1] / csr_col: the neighbourhoods (e.g. from egt_get_csr).
 * The intermediate positions live in a fixed device array of 2^20 float4
 * (16 MB); n above 2^20 is rejected with EGT_ERR_ARG.  Each call first
 * resolves that array's device address (cudaGetSymbolAddress) and loads the
 * half-step kernel on the current device; the first call on a device is the
 * one that commits the 16 MB (held until the process exits) and the kernel's
 * module, so make it before any stream capture.  All calls share the array:
 * calls that may overlap on the GPU race and must be serialised by the
 * caller. */
egt_status egt_taubin_noalloc(const float* pos_in, float* pos_out, const int* csr_off, const int* csr_col,
                              int64_t n, int iters, float lambda, float mu, void* stream);

/* ---- Learned search proposal (no reference counterpart) ------------------
 * A small MLP predicts, per query, a box of grid cells around it (16 classes:
 * 15 boxes of growing size and "plain search") from 8 cell-occupancy
 * features.  The kNN kernel searches the proposed box and keeps its result
 * only when it is certified equal to the plain search's (k-th distance ball
 * inside the box, distinct distances, the plain stop level replayed, no
 * oversized cell); otherwise the plain search runs.  Lists are therefore
 * bit-identical to egt_knn's plain mode whatever the network predicts.
 * Training runs on the device (hand-written forward/backward/Adam kernels,
 * binary16 parameters with FP32 accumulation and FP32 master copies) on labels
 * produced by the plain kNN: the smallest certifying box of each query. */
egt_status egt_proposal_create(int device, int k, uint64_t seed, egt_proposal** out);
void egt_proposal_destroy(egt_proposal* p);
/* Appends the features and labels of every `stride`-th query of h to the
 * training set.  h must hold a plain (or learned) kNN with the proposal's k. */
egt_status egt_proposal_collect(egt_proposal* p, egt_handle* h, int stride);
/* Number of training samples collected so far. */
int64_t egt_proposal_samples(const egt_proposal* p);
/* `steps` Adam steps on mini-batches of `batch` samples drawn with
 * replacement; loss_out (optional, host [steps]) receives each step's mean
 * cross-entropy. */
egt_status egt_proposal_train(egt_proposal* p, int steps, int batch, float lr, float* loss_out);
/* One forward/backward pass over m given samples (host feats [m*8], labels
 * [m]) with the current parameters: grads (host [EGT_PROPOSAL_PARAMS]) of the
 * mean cross-entropy, loss (host, optional).  For gradient checks. */
egt_status egt_proposal_gradients(egt_proposal* p, const float* feats, const uint8_t* labels, int m, float* grads,
                                  float* loss);
/* Parameters as binary16 bit patterns, layout W1[32][8] b1 W2[32][32] b2 W3[16][32] b3. */
egt_status egt_proposal_get_params(const egt_proposal* p, uint16_t* params);
egt_status egt_proposal_set_params(egt_proposal* p, const uint16_t* params);
/* Class choice: the smallest class whose predicted cumulative probability
 * reaches tau (default 0.85). */
egt_status egt_proposal_set_tau(egt_proposal* p, float tau);
float egt_proposal_get_tau(const egt_proposal* p);
/* Autotuner: times the learned kNN on h (which must have been searched with
 * the proposal's k) for each of the ntau thresholds and keeps the fastest;
 * ms_out (optional, host [ntau]) receives the times. */
egt_status egt_proposal_tune(egt_proposal* p, egt_handle* h, const float* taus, int ntau, float* ms_out);
/* Features [n*8], labels [n] (from the handle's last kNN) and proposed
 * classes [n] of every query, sorted space, to host (any may be NULL). */
egt_status egt_proposal_inspect(const egt_proposal* p, egt_handle* h, float* feats, uint8_t* labels,
                                uint8_t* classes);
/* Learned-mode kNN: same outputs as egt_knn (bit-identical lists). */
egt_status egt_knn_learned(egt_handle* h, int k, const egt_proposal* p, void* stream);
/* Makes egt_knn use p when cfg.knn_mode == EGT_KNN_LEARNED (NULL detaches).
 * The proposal must outlive the attachment. */
egt_status egt_attach_proposal(egt_handle* h, const egt_proposal* p);

/* ---- Batched clouds (no reference counterpart) -------------------------------
 * Many independent point clouds through the same path, each with its own k and
 * its own normalisation cube and cell grid exactly as if it were a separate
 * egt_create_cloud handle, so every cloud's lists and positions are identical
 * to that handle's.  Each stage runs as one launch over all clouds: one sort
 * per hierarchy level over (cloud, cell) keys, one persistent kNN kernel
 * claiming query chunks of any cloud, one EGT kernel, and the Taubin loop over
 * the union of the clouds' neighbourhoods as one captured CUDA graph.  An
 * autotuner (first egt_batch_run, cached per size bucket and k) picks the kNN
 * work chunk and the Taubin half-step kernel by timing them on the batch. */
typedef struct egt_batch egt_batch;
typedef struct egt_batch_timings {
    float grid_ms, knn_ms, egt_ms, taubin_ms, output_ms, tune_ms;
    int clouds;
    int64_t points;
    int64_t invalid_queries;  /* over all clouds */
    int64_t exact_reruns;     /* kNN queries re-searched with the one-at-a-time rule */
    int64_t csr_nnz;          /* kept neighbours over all clouds */
    int knn_chunk;            /* queries per work claim (autotuned) */
    int taubin_mode;          /* 0 staged tiles, 1 direct gathers (autotuned) */
    int fused;                /* 1: egt_batch_run ran the kNN and the EGT filter of every cloud in one
                                 persistent launch (knn_ms; k <= 95); egt_ms is then the CSR packing.
                                 The autotuner picks that launch or the two separate ones, whichever
                                 it measured faster: */
    float fused_ms, separate_ms; /* the autotuner's measurements (kNN + filter + CSR), 0 if not run */
} egt_batch_timings;
/* count clouds concatenated in xyz_host ([offsets[count]][3] AoS float),
 * cloud c = points [offsets[c], offsets[c+1]) with k[c] neighbours (1..255). */
egt_status egt_batch_create(const float* xyz_host, const int64_t* offsets, const int* k, int count,
                            const egt_config* cfg, void* stream, egt_batch** out);
egt_status egt_batch_knn(egt_batch* b, void* stream);
egt_status egt_batch_filter(egt_batch* b, float alpha, void* stream);
egt_status egt_batch_taubin(egt_batch* b, int iters, float lambda, float mu, void* stream);
/* Autotune (first call) + kNN + EGT filter + Taubin, always starting from the
 * input positions (the stage calls above work on the current positions). */
egt_status egt_batch_run(egt_batch* b, int iters, float lambda, float mu, float alpha, void* stream);
/* Fixes the tuning (knn_chunk >= 1, taubin_mode 0/1) instead of autotuning. */
egt_status egt_batch_set_tuning(egt_batch* b, int knn_chunk, int taubin_mode);
/* Denormalised positions of all clouds, original order, [offsets[count]][3] AoS host. */
egt_status egt_batch_output(egt_batch* b, float* xyz_host, void* stream);
/* Lists of one cloud like egt_get_knn_host: n_c*k_c ints, original ids and order. */
egt_status egt_batch_get_knn_host(egt_batch* b, int cloud, int* lists_host);
egt_status egt_batch_get_timings(egt_batch* b, egt_batch_timings* t);
void egt_batch_destroy(egt_batch* b);

/* Copies bytes from device memory (e.g. a pointer from egt_get_views) to host
 * memory after synchronising the handle's stream.  No reference counterpart:
 * lets hosts without their own CUDA runtime binding read the device views. */
egt_status egt_copy_to_host(egt_handle* h, void* dst_host, const void* src_dev, int64_t bytes);

/* Number of kernels this library has launched from the calling host thread
 * (all handles).  No reference counterpart: benchmark accounting. */
int64_t egt_kernel_launches(void);

/* ~GridStructure / ~GridMeshCuda: frees every device buffer of the handle. */
void egt_destroy(egt_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* EGT_B200_H */
