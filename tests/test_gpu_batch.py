"""Batched clouds on the GPU (extension; no reference counterpart).

Every cloud of a batch must give exactly what its own GridStructure gives
through the same calls: kNN lists, EGT-filtered lists and smoothed positions,
bit for bit, whatever tuning the batch runs with; and what the CPU oracle (the
restatement of the reference) gives for that cloud alone: identical kNN and EGT
lists, positions within 1e-6 of the bounding-box diagonal of the FP64 oracle.
"""
import numpy as np
import pytest

from golden_util import bbox_diag
from multigpuegtsmoothing_b200 import datagen

pytestmark = pytest.mark.gpu


def _clouds():
    clouds = datagen.batch_clouds(count=14, nmin=2000, nmax=60000, seed=21)
    g = np.random.default_rng(5)
    # edge cases: fewer points than k, a duplicated-point cloud, a lattice
    clouds.append((g.random((7, 3), dtype=np.float32), 10))
    a = g.random((3000, 3), dtype=np.float32)
    clouds.append((np.concatenate([a, a[:300]]), 12))
    t = np.arange(12, dtype=np.float32)
    clouds.append((np.stack(np.meshgrid(t, t, t, indexing="ij"), -1).reshape(-1, 3), 26))
    return clouds


def _single(capi, xyz, k, alpha, iters):
    g = capi.GridStructure(xyz)
    g.GRIDCUDAKNNSELF_COMPACT(k)
    knn = g.GetKNNIndexes()
    e = capi.EGT_CUDA(g)
    e.Filter(alpha)
    filt = g.GetKNNIndexes()
    e.Taubin(iters)
    x, y, z = capi.getOutputPoints(g)
    g.close()
    return knn, filt, np.stack([x, y, z], 1)


@pytest.fixture(scope="module")
def reference(capi):
    clouds = _clouds()
    return clouds, [_single(capi, x, k, 0.65, 20) for x, k in clouds]


def test_batch_stages_match_single_clouds(capi, reference):
    clouds, ref = reference
    b = capi.Batch(clouds)
    b.knn()
    for c, (knn, _, _) in enumerate(ref):
        assert np.array_equal(b.knn_host(c), knn), c
    b.filter(0.65)
    for c, (_, filt, _) in enumerate(ref):
        assert np.array_equal(b.knn_host(c), filt), c
    b.taubin(20)
    out = b.output()
    for c, (_, _, pos) in enumerate(ref):
        assert np.array_equal(out[c], pos), c
    t = b.timings()
    assert t["clouds"] == len(clouds) and t["points"] == sum(x.shape[0] for x, _ in clouds)
    assert t["exact_reruns"] > 0  # the lattice and duplicated clouds tie
    b.close()


@pytest.mark.parametrize("chunk,mode", [(1, 0), (16, 1), (3, 1)])
def test_batch_tuning_does_not_change_results(capi, reference, chunk, mode):
    clouds, ref = reference
    b = capi.Batch(clouds)
    b.set_tuning(chunk, mode)
    b.run(20, 0.63, -0.64, 0.65)
    out = b.output()
    for c, (_, filt, pos) in enumerate(ref):
        assert np.array_equal(b.knn_host(c), filt), c
        assert np.array_equal(out[c], pos), c
    t = b.timings()
    assert t["knn_chunk"] == chunk and t["taubin_mode"] == mode
    b.close()


def test_batch_autotuned_run(capi, reference):
    clouds, ref = reference
    b = capi.Batch(clouds)
    b.run(20, 0.63, -0.64, 0.65)
    out = b.output()
    for c, (_, filt, pos) in enumerate(ref):
        assert np.array_equal(b.knn_host(c), filt), c
        assert np.array_equal(out[c], pos), c
    t = b.timings()
    assert t["knn_chunk"] in (1, 2, 4, 8, 16) and t["taubin_mode"] in (0, 1)
    b.close()


def _original(perm, lists):
    """Sorted-space lists of the oracle in original ids and row order."""
    out = np.full_like(lists, -1)
    out[perm] = np.where(lists >= 0, perm[np.clip(lists, 0, None)], -1)
    return out


def test_batch_clouds_match_oracle(capi, oracle):
    """Clouds of every k in {10, 20, 40} (noisy spheres, the vertices of a
    noisy torus, superquadrics), a lattice (exact ties) and a cloud with
    duplicated points, batched together, each checked against the oracle run on
    that cloud alone."""
    g = np.random.default_rng(9)
    clouds = [(datagen.sphere_cloud(9000, 0.005, 91), 10), (datagen.sphere_cloud(25000, 0.005, 92), 40),
              (datagen.torus_mesh(128, 96)[0], 20),
              (datagen.superquadrics(30000, seed=94), 40)]
    t = np.arange(14, dtype=np.float32)
    clouds.append((np.stack(np.meshgrid(t, t, t, indexing="ij"), -1).reshape(-1, 3), 20))
    a = g.random((5000, 3), dtype=np.float32)
    clouds.append((np.concatenate([a, a[:500]]), 10))
    iters, alpha = 30, 0.65
    b = capi.Batch(clouds)
    b.knn()
    knn = [b.knn_host(c) for c in range(len(clouds))]
    b.filter(alpha)
    filt = [b.knn_host(c) for c in range(len(clouds))]
    b.taubin(iters)
    out = b.output()
    b.close()
    for c, (xyz, k) in enumerate(clouds):
        r = oracle.knn(xyz, k)
        perm = r["perm"]
        assert np.array_equal(knn[c], _original(perm, r["lists"])), c
        e = oracle.egt(r["pos"], r["lists"], alpha)
        assert np.array_equal(filt[c], _original(perm, e)), c
        p64 = oracle.taubin_f64(r["pos"], e, iters)
        lo, hi = float(r["ext"][0]), float(r["ext"][1])
        want = np.empty((xyz.shape[0], 3))
        want[perm] = (p64 * (hi - lo) + lo).T
        assert np.abs(out[c] - want).max() <= 1e-6 * bbox_diag(xyz), c


def test_batch_bad_arguments(capi):
    ok = np.zeros((10, 3), np.float32)
    with pytest.raises(capi.EgtError):
        capi.Batch([(ok, 0)])
    with pytest.raises(capi.EgtError):
        capi.Batch([(ok, 256)])
    with pytest.raises(capi.EgtError):
        capi.Batch([(ok, 10), (np.zeros((0, 3), np.float32), 10)])
    b = capi.Batch([(np.random.default_rng(0).random((100, 3), dtype=np.float32), 5)])
    with pytest.raises(capi.EgtError):
        b.filter(0.65)  # before the kNN
    with pytest.raises(capi.EgtError):
        b.set_tuning(0, 0)
    b.close()


def test_batch_run_is_repeatable(capi, reference):
    clouds, ref = reference
    b = capi.Batch(clouds)
    b.set_tuning(4, 0)
    for _ in range(2):  # each run smooths the input clouds again
        b.run(20, 0.63, -0.64, 0.65)
        out = b.output()
        for c, (_, filt, pos) in enumerate(ref):
            assert np.array_equal(b.knn_host(c), filt), c
            assert np.array_equal(out[c], pos), c
    b.close()
