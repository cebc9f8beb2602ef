// Test-only harness: the reference's own consumers on a provider of this library.
//
// The unmodified reference classes EGT_CUDA (EGT_CUDA.cu), Normal_CUDA
// (Normal_CUDA.cu with CUDA_MST.cu and bfs.cu) and getOutputPoints
// (getOutputPoints.cu), compiled from the reference's sources against its own
// KNNInterface.cuh, run on egtb200::GridStructure / GridMeshCuda through
// egtb200::ReferenceView<::KNNInterface> -- the reference's main.cpp:106-121
// with only the provider replaced.  Their outputs must equal the reference's
// own run (tests/golden fixtures): that is the drop-in contract of
// KNNInterface.  Before the reference's output stage, this library's own runs
// on the same provider, reading what the reference's smoother left in the
// provider's slots.  Built by oracle/ref/Makefile into oracle/_ref/libegtref_consumer.so.
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "KNNInterface.cuh"
#include "EGT_CUDA.cuh"
#include "Normal_CUDA.cuh"
#include "getOutputPoints.cuh"

#include "egt_knn_interface.hpp"

namespace {

void copy_state(::KNNInterface& p, int n, int k, int* lists, float* pos) {
    cudaDeviceSynchronize();
    if (lists) cudaMemcpy(lists, p.GetKNNIndexesInPartitions()[0], sizeof(int) * (size_t)n * k, cudaMemcpyDeviceToHost);
    if (pos) {
        cudaMemcpy(pos, p.GetRefPointsX()[0], sizeof(float) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(pos + n, p.GetRefPointsY()[0], sizeof(float) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(pos + 2 * (size_t)n, p.GetRefPointsZ()[0], sizeof(float) * n, cudaMemcpyDeviceToHost);
    }
}

// The reference's stages on the view, with this library's output stage before the reference's.
int run_consumers(egtb200::Provider& prov, int n, int k, int iters, float alpha, bool normals, int* knn_egt,
                  float* pos_out, float* nrm, float* out_xyz, float* out_xyz_lib) {
    egtb200::ReferenceView<::KNNInterface> view(prov);
    {
        EGT_CUDA smoother(view);
        smoother.PerformSmoothing(iters, 0.63f, -0.64f, alpha);
    }
    copy_state(view, n, k, knn_egt, pos_out);
    if (normals) {
        std::vector<float> nx(n), ny(n), nz(n);
        Normal_CUDA nc(view);
        nc.GetNormals(nx.data(), ny.data(), nz.data());
        if (nrm) {
            std::memcpy(nrm, nx.data(), sizeof(float) * n);
            std::memcpy(nrm + n, ny.data(), sizeof(float) * n);
            std::memcpy(nrm + 2 * (size_t)n, nz.data(), sizeof(float) * n);
        }
    }
    // this library's output stage, reading what the reference's smoother left
    // in the slots; it runs first because the reference's getOutputPoints
    // writes its output back into the provider's position arrays
    // (getOutputPoints.cu:52-58)
    if (out_xyz_lib) {
        egtb200::getOutputPoints(out_xyz_lib, out_xyz_lib + n, out_xyz_lib + 2 * (size_t)n, &prov);
    }
    std::vector<float> ox(n), oy(n), oz(n);
    getOutputPoints(ox.data(), oy.data(), oz.data(), &view);
    if (out_xyz) {
        std::memcpy(out_xyz, ox.data(), sizeof(float) * n);
        std::memcpy(out_xyz + n, oy.data(), sizeof(float) * n);
        std::memcpy(out_xyz + 2 * (size_t)n, oz.data(), sizeof(float) * n);
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

}  // namespace

extern "C" {

// Point cloud: GridStructure(mesh, 1, 1e-6, 1024, 4) + GRIDCUDAKNNSELF_COMPACT(k, 1e8)
// of this library, then the reference's EGT_CUDA / Normal_CUDA / getOutputPoints.
//   knn_egt [n*k], pos_out [3n] (sorted space, after smoothing), normals [3n]
//   (original order), out_xyz [3n] (getOutputPoints of the reference),
//   out_xyz_lib [3n] (this library's getOutputPoints after the reference's smoother).
int egtcons_cloud(const float* xyz, int n, int k, int iters, float alpha, int do_normals, int* knn_egt,
                  float* pos_out, float* normals, float* out_xyz, float* out_xyz_lib) {
    try {
        egtb200::GridStructure grid(xyz, n, 1, 1e-6f, 1024, 4);
        grid.GRIDCUDAKNNSELF_COMPACT(k, 1e8f);
        return run_consumers(grid, n, k, iters, alpha, do_normals != 0, knn_egt, pos_out, normals, out_xyz,
                             out_xyz_lib);
    } catch (const std::exception&) {
        return -1;
    }
}

// Mesh: GridMeshCuda(mesh, 1, 1e-6, 1024) + GetNeighborsFromTriangles(k) of
// this library, then the reference's EGT_CUDA / getOutputPoints.
int egtcons_mesh(const float* xyz, int n, const uint32_t* tris, int t, int k, int iters, float alpha, int* knn_egt,
                 float* pos_out, float* out_xyz, float* out_xyz_lib) {
    try {
        egtb200::GridMeshCuda grid(xyz, n, tris, t, 1, 1e-6f, 1024);
        grid.GetNeighborsFromTriangles(k);
        return run_consumers(grid, n, k, iters, alpha, false, knn_egt, pos_out, nullptr, out_xyz, out_xyz_lib);
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"
