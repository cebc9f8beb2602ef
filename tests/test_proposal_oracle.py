"""CPU checks of the learned-search-proposal oracle (no GPU).

The proposal-driven kNN must return exactly the plain grid kNN's lists for
any per-query class, because a box result is only kept when it is certified
equal to the plain search's; these tests hold the oracle's restatement of
that certification to it on clouds with and without distance ties.  The
network oracle's gradient is checked against finite differences.
"""
import numpy as np
import pytest

from multigpuegtsmoothing_b200 import datagen


def _dense_dups():
    g = np.random.default_rng(1)
    a = (g.random((60000, 3), dtype=np.float32) * np.float32(0.05)).astype(np.float32)
    return np.concatenate([a, a[:6000]])


def _lattice():
    t = np.arange(40, dtype=np.float32)
    return np.stack(np.meshgrid(t, t, t, indexing="ij"), -1).reshape(-1, 3)


@pytest.mark.parametrize("case,k", [("sphere", 40), ("dups", 12), ("lattice", 26)])
def test_proposal_search_equals_plain(oracle, case, k):
    xyz = {"sphere": lambda: datagen.sphere_cloud(), "dups": _dense_dups, "lattice": _lattice}[case]()
    plain = oracle.knn(xyz, k)
    _, labels = oracle.proposal_data(xyz, k)
    n = xyz.shape[0]
    rng = np.random.default_rng(7)
    variants = {
        "labels": labels,
        "under": np.maximum(labels.astype(int) - 1, 0),
        "over": np.minimum(labels.astype(int) + 2, 15),
        "random": rng.integers(0, 16, n),
    }
    for name, cls in variants.items():
        got = oracle.knn_proposal(xyz, k, cls.astype(np.uint8))
        assert np.array_equal(got["lists"], plain["lists"]), (case, name)
        assert np.array_equal(got["level"], plain["level"]), (case, name)
        assert got["invalid"] == plain["invalid"]
        if case == "sphere" and name == "labels":
            # exact labels certify essentially every query
            assert got["certified"].mean() > 0.99
        if name == "under":
            # a box one class smaller than the label never certifies
            assert got["certified"][labels > 0].sum() == 0


def test_proposal_ties_fall_back(oracle):
    # lattice distances repeat: no box result may be accepted
    xyz = _lattice()
    _, labels = oracle.proposal_data(xyz, 26)
    got = oracle.knn_proposal(xyz, 26, labels)
    assert got["certified"].sum() == 0


def test_mlp_oracle_gradient_finite_differences(oracle):
    rng = np.random.default_rng(0)
    p = (rng.standard_normal(1872) * 0.3).astype(np.float64)
    x = rng.random((64, 8))
    y = rng.integers(0, 16, 64)
    _, g = oracle.mlp_loss_grad(p, x, y)
    idx = rng.choice(1872, 60, replace=False)
    eps = 1e-6
    for i in idx:
        e = np.zeros(1872)
        e[i] = eps
        fd = (oracle.mlp_loss_grad(p + e, x, y)[0] - oracle.mlp_loss_grad(p - e, x, y)[0]) / (2 * eps)
        assert abs(fd - g[i]) < 1e-7 + 1e-5 * abs(g[i])


def test_mlp_oracle_classes_monotone_in_tau(oracle):
    rng = np.random.default_rng(1)
    p = (rng.standard_normal(1872) * 0.3).astype(np.float16)
    x = rng.random((500, 8))
    prev = None
    for tau in (0.3, 0.6, 0.9, 1.0):
        c = oracle.mlp_classes(p, x, tau)
        if prev is not None:
            assert np.all(c >= prev)
        prev = c
