"""The C++ adapter (include/egt_knn_interface.hpp) accepts reference-style
caller code: compiled and linked against libegt_b200 with g++, not run (no GPU
here).  The caller uses a mesh type with the reference's Mesh.h layout (the
constructors of GridStructure and GridMeshCuda take it as the reference's do)
and hands the provider, through ReferenceView, to a consumer written against
an abstract class with the reference's KNNInterface.cuh getters."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CALLER = r"""
#include <cstdint>
#include <vector>
// the reference's Mesh.h layout
struct V3 { float x; float y; float z; };
struct I3 { uint32_t v0; uint32_t v1; uint32_t v2; };
struct Mesh { std::vector<V3> mV; std::vector<I3> mF; std::vector<V3> mN; };
// the reference's abstract provider (KNNInterface.cuh:8-31), global namespace
class KNNInterface {
public:
    [[nodiscard]] virtual bool isReady() const = 0;
    [[nodiscard]] virtual int GetNumberOfCards() const = 0;
    virtual float** GetRefPointsX() = 0;
    virtual float** GetRefPointsY() = 0;
    virtual float** GetRefPointsZ() = 0;
    virtual float** GetQuerPointsX() { return GetRefPointsX(); }
    virtual float** GetQuerPointsY() { return GetRefPointsY(); }
    virtual float** GetQuerPointsZ() { return GetRefPointsZ(); }
    virtual int** GetKNNIndexesInPartitions() = 0;
    [[nodiscard]] virtual int GetPartitionSize() const = 0;
    virtual int* GetPointCountInCards() = 0;
    virtual int** GetOriginalRefIndexes() = 0;
    virtual int** GetOriginalQuerIndexes() { return GetOriginalRefIndexes(); }
    virtual void GetKNNIndexes(int* knnIndexes) = 0;
    [[nodiscard]] virtual float GetMaxExtent() const = 0;
    [[nodiscard]] virtual float GetMinExtent() const = 0;
    [[nodiscard]] virtual int pointsRefCount() const = 0;
    [[nodiscard]] virtual int pointsQuerCount() const { return pointsRefCount(); }
    [[nodiscard]] virtual int NeighborCount() const = 0;
};
// a consumer written against it, as the reference's EGT_CUDA is
struct Consumer {
    explicit Consumer(KNNInterface& p) {
        float** x = p.GetRefPointsX();
        int** l = p.GetKNNIndexesInPartitions();
        (void)x; (void)l; (void)p.NeighborCount();
    }
};
#include "egt_knn_interface.hpp"

int main(int argc, char**) {
    if (argc < 100) return 0;  // link check only
    Mesh mesh;
    egtb200::GridStructure grid(mesh, 1, 1e-6, 1024, 4);
    grid.GRIDCUDAKNNSELF_COMPACT(40, 1e8);
    egtb200::ReferenceView<::KNNInterface> view(grid);
    Consumer c(view);
    egtb200::EGT_CUDA(grid).PerformSmoothing(150, 0.63f, -0.64f, 0.65f);
    egtb200::GridMeshCuda m(mesh, 1, 1e-6, 1024);
    m.GetNeighborsFromTriangles(40);
    std::vector<float> x(mesh.mV.size()), y(x), z(x);
    egtb200::getOutputPoints(x.data(), y.data(), z.data(), &m);
    return 0;
}
"""


def test_reference_style_caller_compiles_and_links(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not found")
    lib = os.path.join(ROOT, "multigpuegtsmoothing_b200", "lib")
    if not os.path.exists(os.path.join(lib, "libegt_b200.so")):
        pytest.skip("libegt_b200.so not built")
    src = tmp_path / "caller.cpp"
    src.write_text(CALLER)
    out = tmp_path / "caller"
    r = subprocess.run([gxx, "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                        "-L", lib, "-legt_b200", "-o", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
