"""The reference's CPU normal orienter orient_kruskal (MST.cpp:399-423) on the
GPU, through egt_orient_kruskal.

The oriented normals must equal the reference's own outputs bit for bit on the
golden fixtures (one tree, a forest with empty rows, all-equal weights, and
axis-aligned normals whose exactly-zero dot products stop the sign
propagation), and the CPU oracle's on clouds above 46,340 points, where the
reference's 32-bit edge key would overflow and both use 64-bit keys.
"""
import numpy as np
import pytest

from golden_util import ORIENT, load
from multigpuegtsmoothing_b200 import datagen

pytestmark = pytest.mark.gpu


def _run(capi, knn, nrm, k_use):
    out = np.array(nrm, dtype=np.float32, order="C", copy=True)
    capi.orient_kruskal(knn, out[0], out[1], out[2], k_use=k_use)
    return out


@pytest.mark.parametrize("name", ORIENT)
def test_orient_kruskal_matches_reference(capi, name):
    d, m = load(name)
    got = _run(capi, d["in_knn"], d["in_nrm_in"], m["k_use"])
    assert np.array_equal(got.view(np.uint32), d["ref_nrm_out"].view(np.uint32))


def test_orient_kruskal_large_matches_oracle(capi, oracle):
    kn = oracle.knn(datagen.sphere_cloud(200_000, 0.005, 46), 16)
    nrm = oracle.normals(kn["pos"], kn["lists"])
    rng = np.random.default_rng(47)
    nrm *= np.where(rng.random(nrm.shape[1]) < 0.5, -1.0, 1.0).astype(np.float32)
    lists = kn["lists"].copy()
    lists[rng.random(lists.shape) < 0.3] = -1  # a forest of many trees
    for k_use in (16, 7):
        want = oracle.orient_kruskal(lists, nrm, k_use)
        got = _run(capi, lists, nrm, k_use)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), k_use


def test_orient_kruskal_zero_dot_forest_matches_oracle(capi, oracle):
    """Axis-aligned normals on a larger lattice with blanked entries: many
    trees, each crossing edges with an exactly zero dot product."""
    ax = np.arange(40, dtype=np.float32)
    xyz = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)
    kn = oracle.knn(xyz, 6)
    n = kn["lists"].shape[0]
    rng = np.random.default_rng(48)
    nrm = np.zeros((3, n), np.float32)
    nrm[rng.integers(0, 3, n), np.arange(n)] = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    lists = kn["lists"].copy()
    lists[rng.random(lists.shape) < 0.25] = -1
    want = oracle.orient_kruskal(lists, nrm, 6)
    got = _run(capi, lists, nrm, 6)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_orient_kruskal_rejects_bad_input(capi):
    knn = np.array([[1, 2], [0, 5], [0, 1]], np.int32)  # 5 >= n
    nx, ny, nz = (np.ones(3, np.float32) for _ in range(3))
    with pytest.raises(capi.EgtError):
        capi.orient_kruskal(knn, nx, ny, nz, k_use=2)
    with pytest.raises(capi.EgtError):
        capi.orient_kruskal(knn, nx, ny, nz, k_use=3)  # k_use > k
    # k_use = 1 never reads the bad entry
    capi.orient_kruskal(knn, nx, ny, nz, k_use=1)


CPP_CALLER = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "egt_knn_interface.hpp"
int main(int argc, char** argv) {
    const int n = std::atoi(argv[1]), k = std::atoi(argv[2]), k_use = std::atoi(argv[3]);
    std::vector<int> knn((size_t)n * k);
    std::vector<float> nrm((size_t)3 * n);
    FILE* f = std::fopen(argv[4], "rb");
    if (!f || std::fread(knn.data(), 4, knn.size(), f) != knn.size() ||
        std::fread(nrm.data(), 4, nrm.size(), f) != nrm.size()) return 2;
    std::fclose(f);
    egtb200::orient_kruskal(knn.data(), nrm.data(), nrm.data() + n, nrm.data() + 2 * n, nullptr, nullptr,
                            nullptr, n, k, k_use);
    f = std::fopen(argv[5], "wb");
    if (!f || std::fwrite(nrm.data(), 4, nrm.size(), f) != nrm.size()) return 3;
    std::fclose(f);
    return 0;
}
"""


def test_cpp_adapter_orient_kruskal(tmp_path):
    """A C++ caller of the reference's free function, switched to the adapter
    header (include/egt_knn_interface.hpp), gets the reference's normals."""
    import os
    import shutil
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    lib = os.path.join(root, "multigpuegtsmoothing_b200", "lib")
    src = tmp_path / "caller.cpp"
    src.write_text(CPP_CALLER)
    exe = tmp_path / "caller"
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", os.path.join(root, "include"), str(src), "-L", lib,
                    "-legt_b200", f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    d, m = load("ref_orient_forest")
    knn = np.ascontiguousarray(d["in_knn"], dtype=np.int32)
    nrm = np.ascontiguousarray(d["in_nrm_in"], dtype=np.float32)
    n, k = knn.shape
    (tmp_path / "in.bin").write_bytes(knn.tobytes() + nrm.tobytes())
    subprocess.run([str(exe), str(n), str(k), str(m["k_use"]), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")],
                   check=True)
    got = np.frombuffer((tmp_path / "out.bin").read_bytes(), dtype=np.uint32).reshape(3, n)
    assert np.array_equal(got, d["ref_nrm_out"].view(np.uint32))
