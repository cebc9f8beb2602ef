// Test-only harness around the UNMODIFIED reference implementation.
//
// This file is oracle infrastructure: it is compiled together with the
// reference's own CUDA sources (GridKNNCuda.cu, GridMeshCuda1.cu, EGT_CUDA.cu,
// Normal_CUDA.cu, CUDA_MST.cu, bfs.cu, getOutputPoints.cu) by oracle/ref/Makefile
// into oracle/_ref/libegtref.so.  It drives the reference exactly the way the
// reference CLI does (main.cpp:106-121) and copies out the intermediate device
// buffers so that tests can pin the CPU oracle and the product kernels against
// the reference itself.  Nothing in the product links or loads this library.
//
// Sequence reproduced (reference main.cpp:106-121):
//   cloud: GridStructure(mesh, 1, 1e-6, 1024, 4) -> GRIDCUDAKNNSELF_COMPACT(k, 1e8)
//          -> EGT_CUDA::PerformSmoothing(iters, 0.63, -0.64, alpha)
//          -> Normal_CUDA::GetNormals -> getOutputPoints
//   mesh:  GridMeshCuda(mesh, 1, 1e-6, 1024) -> GetNeighborsFromTriangles(k)
//          -> PerformSmoothing -> getOutputPoints
//   query: GridStructure(ref) -> GRIDCUDAKNNCompact(queries) -> GetKNNIndexes
// The only addition is that every stage is bracketed by cudaEvents and the
// intermediate device arrays are copied to host buffers supplied by the caller.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>
#include <cuda_runtime.h>

#include "Mesh.h"
#include "KNNInterface.cuh"
#include "GridKNNCuda.cuh"
#include "GridMeshCuda1.cuh"
#include "EGT_CUDA.cuh"
#include "Normal_CUDA.cuh"
#include "getOutputPoints.cuh"

namespace {

struct StageTimer {
    cudaEvent_t a{}, b{};
    StageTimer() { cudaEventCreate(&a); cudaEventCreate(&b); }
    ~StageTimer() { cudaEventDestroy(a); cudaEventDestroy(b); }
    void start() { cudaDeviceSynchronize(); cudaEventRecord(a); }
    float stop() {
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    }
};

void copy_sorted_positions(KNNInterface& prov, int n, float* dst) {
    if (!dst) return;
    cudaMemcpy(dst, prov.GetRefPointsX()[0], sizeof(float) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(dst + n, prov.GetRefPointsY()[0], sizeof(float) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(dst + 2 * (size_t)n, prov.GetRefPointsZ()[0], sizeof(float) * n, cudaMemcpyDeviceToHost);
}

void copy_lists(KNNInterface& prov, int n, int k, int* dst) {
    if (!dst) return;
    cudaMemcpy(dst, prov.GetKNNIndexesInPartitions()[0], sizeof(int) * (size_t)n * k,
               cudaMemcpyDeviceToHost);
}

int finish(const char* where) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "egtref: CUDA error after %s: %s\n", where, cudaGetErrorString(e));
        return -1;
    }
    return 0;
}

Mesh make_mesh(const float* xyz, int n, const uint32_t* tris, int t) {
    Mesh m;
    m.mV.resize(n);
    for (int i = 0; i < n; i++) m.mV[i] = V3{xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2]};
    if (tris) {
        m.mF.resize(t);
        for (int i = 0; i < t; i++)
            m.mF[i] = I3{tris[3 * (size_t)i], tris[3 * (size_t)i + 1], tris[3 * (size_t)i + 2]};
    }
    return m;
}

}  // namespace

extern "C" {

// Point-cloud pipeline.  All output pointers are optional (may be null).
//   knn_raw   [n*k]  sorted-space lists right after GRIDCUDAKNNSELF_COMPACT
//   knn_egt   [n*k]  sorted-space lists after the in-place EGT filter
//   pos_in    [3n]   SoA, normalised, sorted space, before smoothing
//   pos_out   [3n]   SoA, normalised, sorted space, after smoothing
//   perm      [n]    sorted slot -> original index
//   extents   [2]    {min, max} of the normalisation cube
//   normals   [3n]   SoA, original order (only when do_normals != 0)
//   out_xyz   [3n]   SoA, original order, denormalised (getOutputPoints)
//   stage_ms  [4]    {grid+kNN, EGT+Taubin, normals, output}
int egtref_cloud(const float* xyz, int n, int k, int iters, float alpha, int do_normals,
                 int* knn_raw, int* knn_egt, float* pos_in, float* pos_out, int* perm,
                 float* extents, float* normals, float* out_xyz, float* stage_ms) {
    cudaSetDevice(0);
    Mesh mesh = make_mesh(xyz, n, nullptr, 0);
    StageTimer tm;
    float ms[4] = {0, 0, 0, 0};
    tm.start();
    auto grid = std::make_shared<GridStructure>(mesh, 1, 1e-6, 1024, 4);
    grid->GRIDCUDAKNNSELF_COMPACT(k, 1e8);
    ms[0] = tm.stop();
    if (finish("knn")) return -1;
    copy_lists(*grid, n, k, knn_raw);
    copy_sorted_positions(*grid, n, pos_in);
    if (perm) cudaMemcpy(perm, grid->GetOriginalRefIndexes()[0], sizeof(int) * n, cudaMemcpyDeviceToHost);
    if (extents) { extents[0] = grid->GetMinExtent(); extents[1] = grid->GetMaxExtent(); }

    tm.start();
    {
        EGT_CUDA smoother(*grid);
        smoother.PerformSmoothing(iters, 0.63, -0.64, alpha);
    }
    ms[1] = tm.stop();
    if (finish("smoothing")) return -1;
    copy_lists(*grid, n, k, knn_egt);
    copy_sorted_positions(*grid, n, pos_out);

    if (do_normals) {
        std::vector<float> nx(n), ny(n), nz(n);
        tm.start();
        Normal_CUDA nc(*grid);
        nc.GetNormals(nx.data(), ny.data(), nz.data());
        ms[2] = tm.stop();
        if (finish("normals")) return -1;
        if (normals) {
            std::memcpy(normals, nx.data(), sizeof(float) * n);
            std::memcpy(normals + n, ny.data(), sizeof(float) * n);
            std::memcpy(normals + 2 * (size_t)n, nz.data(), sizeof(float) * n);
        }
    }
    {
        std::vector<float> ox(n), oy(n), oz(n);
        tm.start();
        getOutputPoints(ox.data(), oy.data(), oz.data(), grid.get());
        ms[3] = tm.stop();
        if (finish("output")) return -1;
        if (out_xyz) {
            std::memcpy(out_xyz, ox.data(), sizeof(float) * n);
            std::memcpy(out_xyz + n, oy.data(), sizeof(float) * n);
            std::memcpy(out_xyz + 2 * (size_t)n, oz.data(), sizeof(float) * n);
        }
    }
    if (stage_ms) for (int i = 0; i < 4; i++) stage_ms[i] = ms[i];
    return 0;
}

// Mesh pipeline (no normals, as in the reference CLI).  Same output conventions;
// stage_ms = {grid+1-ring, EGT+Taubin, 0, output}.
int egtref_mesh(const float* xyz, int n, const uint32_t* tris, int t, int k, int iters, float alpha,
                int* knn_raw, int* knn_egt, float* pos_in, float* pos_out, int* perm,
                float* extents, float* out_xyz, float* stage_ms) {
    cudaSetDevice(0);
    Mesh mesh = make_mesh(xyz, n, tris, t);
    StageTimer tm;
    float ms[4] = {0, 0, 0, 0};
    tm.start();
    auto grid = std::make_shared<GridMeshCuda>(mesh, 1, 1e-6, 1024);
    grid->GetNeighborsFromTriangles(k);
    ms[0] = tm.stop();
    if (finish("mesh 1-ring")) return -1;
    copy_lists(*grid, n, k, knn_raw);
    copy_sorted_positions(*grid, n, pos_in);
    if (perm) cudaMemcpy(perm, grid->GetOriginalRefIndexes()[0], sizeof(int) * n, cudaMemcpyDeviceToHost);
    if (extents) { extents[0] = grid->GetMinExtent(); extents[1] = grid->GetMaxExtent(); }
    tm.start();
    {
        EGT_CUDA smoother(*grid);
        smoother.PerformSmoothing(iters, 0.63, -0.64, alpha);
    }
    ms[1] = tm.stop();
    if (finish("smoothing")) return -1;
    copy_lists(*grid, n, k, knn_egt);
    copy_sorted_positions(*grid, n, pos_out);
    {
        std::vector<float> ox(n), oy(n), oz(n);
        tm.start();
        getOutputPoints(ox.data(), oy.data(), oz.data(), grid.get());
        ms[3] = tm.stop();
        if (finish("output")) return -1;
        if (out_xyz) {
            std::memcpy(out_xyz, ox.data(), sizeof(float) * n);
            std::memcpy(out_xyz + n, oy.data(), sizeof(float) * n);
            std::memcpy(out_xyz + 2 * (size_t)n, oz.data(), sizeof(float) * n);
        }
    }
    if (stage_ms) for (int i = 0; i < 4; i++) stage_ms[i] = ms[i];
    return 0;
}

// Query-vs-reference kNN, the reference's other search (ICP use):
// GridStructure(ref) -> GRIDCUDAKNNCompact(qx, qy, qz, nq, k, 1e8)
// (GridKNNCuda.cu:1645-1939) -> GetKNNIndexes (:1941-1968).
//   q        [nq*3] AoS query points (the reference's units)
//   knn      [nq*k] original reference ids in original query order
//   stage_ms [1]    {grid + query kNN}
int egtref_query(const float* xyz, int n, const float* q, int nq, int k, int* knn, float* stage_ms) {
    cudaSetDevice(0);
    Mesh mesh = make_mesh(xyz, n, nullptr, 0);
    std::vector<float> qx(nq), qy(nq), qz(nq);
    for (int i = 0; i < nq; i++) {
        qx[i] = q[3 * (size_t)i];
        qy[i] = q[3 * (size_t)i + 1];
        qz[i] = q[3 * (size_t)i + 2];
    }
    StageTimer tm;
    tm.start();
    auto grid = std::make_shared<GridStructure>(mesh, 1, 1e-6, 1024, 4);
    grid->GRIDCUDAKNNCompact(qx.data(), qy.data(), qz.data(), nq, k, 1e8);
    const float ms = tm.stop();
    if (finish("query knn")) return -1;
    grid->GetKNNIndexes(knn);
    if (finish("GetKNNIndexes")) return -1;
    if (stage_ms) stage_ms[0] = ms;
    return 0;
}

}  // extern "C"
