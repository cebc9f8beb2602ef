"""Seeded synthetic inputs for the point-cloud / mesh smoothing workloads.

The reference ships no sample data (its four scans are missing from the
repository), so every workload is generated here from a seed with numpy's
PCG64 generator.  Each generator returns float32 arrays in original (unsorted)
point order, the layout the reference reads from a PLY file (``Mesh.mV``,
reference Mesh.h:34-50): ``xyz`` is an (N, 3) float32 AoS array and ``tris`` an
(T, 3) uint32 array of vertex indices.

Workloads (sizes are the ones the benchmarks and parity tests use):

* ``sphere_cloud``    noisy unit sphere, N=35,947, sigma=0.005 (radial).
* ``torus_mesh``      torus R=1, r=0.3 on a 512x256 grid -> 131,072 vertices,
                      262,144 triangles, isotropic noise sigma=0.5% of r.
* ``superquadrics``   4M points on three overlapping superellipsoids with a
                      50:1 clustered density and noise 0.2% of the bbox diagonal.
* ``batch_clouds``    256 clouds, N log-uniform in [2K, 500K], k in {10,20,40},
                      each a noisy sphere or torus sample.
* ``sheets``          20M points, Gaussian-thickened planar and spherical sheets
                      with a 1000:1 density range (learned-proposal workload).
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "sphere_cloud",
    "torus_mesh",
    "superquadrics",
    "batch_clouds",
    "sheets",
]


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def sphere_cloud(n: int = 35947, sigma: float = 0.005, seed: int = 1) -> np.ndarray:
    """Points uniform on the unit sphere, displaced radially by N(0, sigma)."""
    g = _rng(seed)
    d = g.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = 1.0 + sigma * g.standard_normal(n)
    return (d * r[:, None]).astype(np.float32)


def torus_mesh(nu: int = 512, nv: int = 256, R: float = 1.0, r: float = 0.3,
               noise_frac: float = 0.005, seed: int = 2):
    """Parametric torus triangulated on an nu x nv grid.

    Vertex (i, j) has index i*nv + j, u = 2*pi*i/nu, v = 2*pi*j/nv.  Each grid
    quad (i,j),(i+1,j),(i+1,j+1),(i,j+1) (indices wrap) is split into the two
    triangles (a,b,c) and (a,c,d).  Isotropic Gaussian noise of std
    noise_frac*r is added to every vertex.
    """
    g = _rng(seed)
    i = np.arange(nu)[:, None]
    j = np.arange(nv)[None, :]
    u = 2.0 * np.pi * i / nu
    v = 2.0 * np.pi * j / nv
    x = (R + r * np.cos(v)) * np.cos(u)
    y = (R + r * np.cos(v)) * np.sin(u)
    z = np.broadcast_to(r * np.sin(v), x.shape)
    xyz = np.stack([x, y, z], axis=-1).reshape(-1, 3)
    xyz = xyz + noise_frac * r * g.standard_normal(xyz.shape)
    ii, jj = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    a = ii * nv + jj
    b = ((ii + 1) % nu) * nv + jj
    c = ((ii + 1) % nu) * nv + (jj + 1) % nv
    d = ii * nv + (jj + 1) % nv
    t1 = np.stack([a, b, c], axis=-1).reshape(-1, 3)
    t2 = np.stack([a, c, d], axis=-1).reshape(-1, 3)
    tris = np.empty((2 * nu * nv, 3), dtype=np.uint32)
    tris[0::2] = t1
    tris[1::2] = t2
    return xyz.astype(np.float32), tris


def _spow(base: np.ndarray, e: float) -> np.ndarray:
    return np.sign(base) * np.abs(base) ** e


def _superellipsoid(g: np.random.Generator, m: int, e1: float, e2: float,
                    scale, centre) -> np.ndarray:
    eta = g.uniform(-np.pi / 2, np.pi / 2, m)
    om = g.uniform(-np.pi, np.pi, m)
    ce, se = np.cos(eta), np.sin(eta)
    x = _spow(ce, e1) * _spow(np.cos(om), e2)
    y = _spow(ce, e1) * _spow(np.sin(om), e2)
    z = _spow(se, e1)
    p = np.stack([x, y, z], axis=1) * np.asarray(scale)[None, :]
    return p + np.asarray(centre)[None, :]


def superquadrics(n: int = 4_000_000, density_ratio: float = 50.0,
                  noise_frac: float = 0.002, seed: int = 3) -> np.ndarray:
    """n points on three overlapping superellipsoids, clustered density.

    Surface samples (parametric) are accepted with probability
    rho(p)/rho_max where rho = 1 + (ratio-1) * max_c exp(-|p-c|^2 / 2s^2) over
    12 seeded Gaussian cluster centres, so the densest regions are `ratio`
    times denser than the sparsest.  Noise std = noise_frac * bbox diagonal.
    """
    g = _rng(seed)
    shapes = [
        ((0.3, 0.3), (1.0, 0.8, 0.6), (-0.35, 0.0, 0.0)),
        ((1.0, 1.0), (0.7, 0.7, 0.7), (0.35, 0.1, 0.05)),
        ((2.0, 0.5), (0.6, 0.9, 0.5), (0.0, -0.3, 0.2)),
    ]
    centres = g.uniform(-0.9, 0.9, (12, 3)).astype(np.float32)
    inv_s2 = np.float32(1.0 / (2.0 * 0.18 ** 2))
    out = []
    have = 0
    while have < n:
        m = 1 << 21
        which = g.integers(0, 3, m)
        pts = np.empty((m, 3), dtype=np.float32)
        for s, (ee, sc, c0) in enumerate(shapes):
            sel = which == s
            pts[sel] = _superellipsoid(g, int(sel.sum()), ee[0], ee[1], sc, c0)
        # squared distance to every cluster centre via |p|^2 - 2 p.c + |c|^2
        d2 = (np.sum(pts * pts, axis=1, keepdims=True) - 2.0 * pts @ centres.T
              + np.sum(centres * centres, axis=1)[None, :])
        best = np.exp(-np.min(d2, axis=1) * inv_s2)
        rho = 1.0 + (density_ratio - 1.0) * best
        keep = g.uniform(0.0, density_ratio, m).astype(np.float32) < rho
        pts = pts[keep]
        out.append(pts[: n - have].astype(np.float64))
        have += len(out[-1])
    p = np.concatenate(out)[:n]
    diag = float(np.linalg.norm(p.max(0) - p.min(0)))
    p = p + noise_frac * diag * g.standard_normal(p.shape)
    return p.astype(np.float32)


def batch_clouds(count: int = 256, nmin: int = 2000, nmax: int = 500_000, seed: int = 4):
    """`count` independent clouds: list of (xyz float32 (N,3), k) pairs.

    N is log-uniform in [nmin, nmax], k uniform in {10, 20, 40}; each cloud is
    a noisy sphere (sigma 0.005) or a noisy torus sample (R=1, r=0.3, sigma
    0.5% of r), picked with probability 1/2, with a random offset and scale.
    """
    g = _rng(seed)
    out = []
    for _ in range(count):
        n = int(np.exp(g.uniform(np.log(nmin), np.log(nmax))))
        k = int(g.choice([10, 20, 40]))
        sub = int(g.integers(0, 2**31 - 1))
        if g.uniform() < 0.5:
            xyz = sphere_cloud(n, 0.005, sub)
        else:
            gg = _rng(sub)
            u = gg.uniform(0, 2 * np.pi, n)
            v = gg.uniform(0, 2 * np.pi, n)
            x = (1.0 + 0.3 * np.cos(v)) * np.cos(u)
            y = (1.0 + 0.3 * np.cos(v)) * np.sin(u)
            z = 0.3 * np.sin(v)
            xyz = np.stack([x, y, z], 1) + 0.0015 * gg.standard_normal((n, 3))
            xyz = xyz.astype(np.float32)
        xyz = (xyz * np.float32(g.uniform(0.5, 4.0)) +
               g.uniform(-10, 10, 3).astype(np.float32)).astype(np.float32)
        out.append((xyz, k))
    return out


def sheets(n: int = 20_000_000, density_range: float = 1000.0, seed: int = 5,
           chunk: int = 1 << 22) -> np.ndarray:
    """n points on Gaussian-thickened planar and spherical sheets.

    Four planes and three spheres; along each sheet the sampling density is
    modulated by a smooth field exp(c * f) with f in [0,1] chosen so the
    densest to sparsest ratio is `density_range`.  Thickness std is 0.002.
    """
    g = _rng(seed)
    planes = [  # (origin, normal axis pair spanning the plane)
        ((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0)),
        ((0.0, 0.0, 0.3), (1.0, 0.0, 0.0), (0.0, 0.6, 0.8)),
        ((0.2, -0.1, -0.2), (0.0, 0.0, 1.0), (0.8, 0.6, 0.0)),
        ((-0.3, 0.3, 0.0), (0.6, -0.8, 0.0), (0.0, 0.0, 1.0)),
    ]
    spheres = [((0.3, 0.3, 0.3), 0.35), ((-0.4, -0.2, 0.1), 0.25), ((0.1, -0.4, -0.3), 0.2)]
    log_r = np.log(density_range)
    out = []
    have = 0
    while have < n:
        m = min(chunk, 4 * (n - have))
        kind = g.integers(0, len(planes) + len(spheres), m)
        pts = np.empty((m, 3))
        for s, (o, a, b) in enumerate(planes):
            sel = kind == s
            c = int(sel.sum())
            uv = g.uniform(-0.8, 0.8, (c, 2))
            pts[sel] = np.asarray(o) + uv[:, :1] * np.asarray(a) + uv[:, 1:] * np.asarray(b)
        for s, (c0, rad) in enumerate(spheres):
            sel = kind == len(planes) + s
            c = int(sel.sum())
            d = g.standard_normal((c, 3))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            pts[sel] = np.asarray(c0) + rad * d
        f = 0.5 + 0.5 * np.sin(3.0 * pts[:, 0] + 1.0) * np.cos(2.0 * pts[:, 1] - 0.5)
        accept = g.uniform(0.0, 1.0, m) < np.exp(log_r * (f - 1.0))
        pts = pts[accept]
        pts = pts + 0.002 * g.standard_normal(pts.shape)
        take = pts[: n - have]
        out.append(take.astype(np.float32))
        have += len(take)
    return np.concatenate(out)[:n]
