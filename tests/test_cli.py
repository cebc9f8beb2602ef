"""The KNNCUDA command line: PLY input/output (CPU) and the full pipeline (GPU)
against the Python mirror of the same call sequence."""
import os
import struct
import subprocess

import numpy as np
import pytest

from multigpuegtsmoothing_b200 import datagen

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(os.path.dirname(HERE), "multigpuegtsmoothing_b200", "bin", "KNNCUDA")


def write_ply(path, xyz, tris=None, ascii=False, rgb=None, big_endian=False):
    n = len(xyz)
    hdr = ["ply", "format " + ("ascii" if ascii else ("binary_big_endian" if big_endian else "binary_little_endian"))
           + " 1.0", f"element vertex {n}", "property double x", "property double y", "property double z"]
    if rgb is not None:
        hdr += ["property uchar red", "property uchar green", "property uchar blue"]
    if tris is not None:
        hdr += [f"element face {len(tris)}", "property list uchar int vertex_indices"]
    hdr.append("end_header")
    with open(path, "wb") as f:
        f.write(("\n".join(hdr) + "\n").encode())
        e = ">" if big_endian else "<"
        for i in range(n):
            if ascii:
                s = " ".join(repr(float(v)) for v in xyz[i])
                if rgb is not None:
                    s += " " + " ".join(str(int(c)) for c in rgb[i])
                f.write((s + "\n").encode())
            else:
                f.write(struct.pack(e + "ddd", *map(float, xyz[i])))
                if rgb is not None:
                    f.write(bytes(int(c) for c in rgb[i]))
        if tris is not None:
            for t in tris:
                if ascii:
                    f.write(("3 " + " ".join(str(int(v)) for v in t) + "\n").encode())
                else:
                    f.write(struct.pack(e + "Biii", 3, *map(int, t)))


def read_out_ply(path):
    """Parses the reference's output layout (binary little-endian)."""
    data = open(path, "rb").read()
    end = data.index(b"end_header\n") + len(b"end_header\n")
    hdr = data[:end].decode().splitlines()
    nv = int([l for l in hdr if l.startswith("element vertex")][0].split()[-1])
    nf_l = [l for l in hdr if l.startswith("element face")]
    nf = int(nf_l[0].split()[-1]) if nf_l else 0
    props = [l.split()[-1] for l in hdr if l.startswith("property") and "list" not in l]
    vprops = props[: props.index("blue") + 1] if "blue" in props else props
    fmt = "".join("f" if p in ("x", "y", "z", "nx", "ny", "nz") else "B" for p in vprops)
    rec = struct.calcsize("<" + fmt)
    V = np.zeros((nv, len(vprops)), np.float64)
    off = end
    for i in range(nv):
        V[i] = struct.unpack_from("<" + fmt, data, off)
        off += rec
    F = np.zeros((nf, 3), np.int64)
    for i in range(nf):
        c, a, b, d = struct.unpack_from("<BIII", data, off)
        assert c == 3
        F[i] = (a, b, d)
        off += 13
    return vprops, V, F


@pytest.mark.parametrize("ascii,big", [(False, False), (True, False), (False, True)])
def test_ply_roundtrip(tmp_path, ascii, big):
    xyz = datagen.sphere_cloud(500, 0.01, 3).astype(np.float64)
    tris = np.array([[0, 1, 2], [2, 3, 4], [5, 6, 7]])
    rgb = np.random.default_rng(0).integers(0, 255, (500, 3))
    src = tmp_path / "in.ply"
    write_ply(str(src), xyz, tris, ascii=ascii, rgb=rgb, big_endian=big)
    dst = tmp_path / "out.ply"
    subprocess.run([BIN, "--ply-roundtrip", str(src), str(dst)], check=True)
    props, V, F = read_out_ply(str(dst))
    assert props == ["x", "y", "z", "red", "green", "blue"]
    assert np.array_equal(V[:, :3], xyz.astype(np.float32).astype(np.float64))
    assert np.array_equal(V[:, 3:].astype(int), rgb)
    assert np.array_equal(F, tris)


@pytest.mark.parametrize("layout", ["le_float", "be_double", "ascii_lines", "ascii_split", "quads", "ascii_quads"])
def test_ply_large_inputs(tmp_path, layout):
    """Inputs large enough for the parallel decoders (fixed-size binary
    records, one ASCII record per line, all-triangle face lists), and the
    layouts that fall back to the sequential reader (records split over
    lines, polygons other than triangles); every one must read the same
    values."""
    rng = np.random.default_rng(7)
    n, nf = 200_003, 150_001
    xyz = rng.normal(size=(n, 3)) * 50.0
    rgb = rng.integers(0, 256, (n, 3))
    tris = rng.integers(0, n, (nf, 3))
    src = tmp_path / "big.ply"
    if layout == "le_float":
        xyz = xyz.astype(np.float32).astype(np.float64)
        hdr = (f"ply\nformat binary_little_endian 1.0\nelement vertex {n}\nproperty float x\nproperty float y\n"
               f"property float z\nproperty uchar red\nproperty uchar green\nproperty uchar blue\n"
               f"element face {nf}\nproperty list uchar int vertex_indices\nend_header\n")
        rec = np.zeros(n, dtype=[("p", "<f4", 3), ("c", "u1", 3)])
        rec["p"] = xyz
        rec["c"] = rgb
        frec = np.zeros(nf, dtype=[("k", "u1"), ("i", "<i4", 3)])
        frec["k"] = 3
        frec["i"] = tris
        src.write_bytes(hdr.encode() + rec.tobytes() + frec.tobytes())
    elif layout in ("be_double", "quads"):
        hdr = (f"ply\nformat binary_big_endian 1.0\nelement vertex {n}\nproperty double x\nproperty short s\n"
               f"property double y\nproperty double z\nproperty uchar red\nproperty uchar green\n"
               f"property uchar blue\nelement face {nf}\nproperty list uchar uint vertex_indices\nend_header\n")
        rec = np.zeros(n, dtype=[("x", ">f8"), ("s", ">i2"), ("y", ">f8"), ("z", ">f8"), ("c", "u1", 3)])
        rec["x"], rec["y"], rec["z"] = xyz[:, 0], xyz[:, 1], xyz[:, 2]
        rec["c"] = rgb
        if layout == "be_double":
            frec = np.zeros(nf, dtype=[("k", "u1"), ("i", ">u4", 3)])
            frec["k"] = 3
            frec["i"] = tris
            body = frec.tobytes()
        else:  # every fifth face is a quad: its first three indices are kept
            parts = []
            for j, t in enumerate(tris):
                if j % 5 == 0:
                    parts.append(struct.pack(">B4I", 4, *map(int, t), 0))
                else:
                    parts.append(struct.pack(">B3I", 3, *map(int, t)))
            body = b"".join(parts)
        src.write_bytes(hdr.encode() + rec.tobytes() + body)
    else:
        hdr = (f"ply\nformat ascii 1.0\ncomment generated\nelement vertex {n}\nproperty double x\n"
               f"property double y\nproperty double z\nproperty uchar red\nproperty uchar green\n"
               f"property uchar blue\nelement face {nf}\nproperty list uchar int vertex_indices\nend_header\n")
        lines = [f"{a!r} {b!r} {c!r} {r} {g} {bb}" for (a, b, c), (r, g, bb) in zip(xyz.tolist(), rgb.tolist())]
        if layout == "ascii_split":  # a record spread over two lines
            lines[n // 2] = lines[n // 2].replace(" ", "\n", 1)
        faces = [f"3 {a} {b} {c}" for a, b, c in tris.tolist()]
        if layout == "ascii_quads":  # every fifth face a quad: its first three indices are kept
            faces = [f"4 {a} {b} {c} 0" if j % 5 == 0 else f"3 {a} {b} {c}"
                     for j, (a, b, c) in enumerate(tris.tolist())]
        src.write_bytes((hdr + "\n".join(lines) + "\n" + "\n".join(faces) + "\n").encode())
    dst = tmp_path / "out.ply"
    subprocess.run([BIN, "--ply-roundtrip", str(src), str(dst)], check=True)
    data = dst.read_bytes()
    end = data.index(b"end_header\n") + len(b"end_header\n")
    out = np.frombuffer(data, dtype=[("p", "<f4", 3), ("c", "u1", 3)], count=n, offset=end)
    assert np.array_equal(out["p"], xyz.astype(np.float32))
    assert np.array_equal(out["c"].astype(np.int64), rgb)
    fo = np.frombuffer(data, dtype=[("k", "u1"), ("i", "<u4", 3)], count=nf, offset=end + n * 15)
    assert np.all(fo["k"] == 3)
    assert np.array_equal(fo["i"].astype(np.int64), tris)


def test_ply_rejects_truncated_data(tmp_path):
    n = 100_000
    hdr = (f"ply\nformat binary_little_endian 1.0\nelement vertex {n}\nproperty float x\nproperty float y\n"
           f"property float z\nelement face 10\nproperty list uchar int vertex_indices\nend_header\n").encode()
    body = np.zeros(3 * n, np.float32).tobytes() + b"".join(struct.pack("<B3i", 3, 0, 1, 2) for _ in range(10))
    for cut, what in [(len(hdr) - 5, b"end_header"), (len(hdr) + 1000, b"truncated vertex"),
                      (len(hdr) + len(body) - 1, b"truncated face")]:
        src = tmp_path / "cut.ply"
        src.write_bytes((hdr + body)[:cut])
        r = subprocess.run([BIN, "--ply-roundtrip", str(src), str(tmp_path / "o.ply")], capture_output=True)
        assert r.returncode != 0 and what in r.stderr, (cut, r.stderr)


def test_cli_rejects_bad_arguments(tmp_path):
    r = subprocess.run([BIN], capture_output=True)
    assert r.returncode != 0 and b"usage" in r.stderr
    src = tmp_path / "in.ply"
    write_ply(str(src), datagen.sphere_cloud(100, 0.01, 3))
    r = subprocess.run([BIN, str(src), "10", "5", "0.65", "0", "2"], capture_output=True, cwd=tmp_path)
    assert r.returncode != 0 and b"ncards must be 1" in r.stderr


@pytest.mark.gpu
def test_cli_cloud_matches_api(tmp_path, capi):
    xyz = datagen.sphere_cloud(6000, 0.005, 5)
    src = tmp_path / "cloud.ply"
    write_ply(str(src), xyz)
    r = subprocess.run([BIN, str(src), "16", "5", "0.65", "0", "1"], capture_output=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert b"Succeeded!" in r.stdout
    props, V, _ = read_out_ply(str(tmp_path / "output.ply"))
    assert props == ["x", "y", "z", "nx", "ny", "nz"]
    g = capi.GridStructure(xyz.astype(np.float32))
    g.GRIDCUDAKNNSELF_COMPACT(16)
    capi.EGT_CUDA(g).PerformSmoothing(5, 0.63, -0.64, 0.65)
    nx, ny, nz = capi.Normal_CUDA(g).GetNormals()
    x, y, z = capi.getOutputPoints(g)
    assert np.array_equal(V[:, 0:3].astype(np.float32), np.stack([x, y, z], 1))
    assert np.array_equal(V[:, 3:6].astype(np.float32), np.stack([nx, ny, nz], 1))


@pytest.mark.gpu
def test_cli_mesh_matches_api(tmp_path, capi):
    xyz, tris = datagen.torus_mesh(64, 32, seed=6)
    src = tmp_path / "mesh.ply"
    write_ply(str(src), xyz, tris)
    r = subprocess.run([BIN, str(src), "40", "5", "1e-8", "1", "1"], capture_output=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    props, V, F = read_out_ply(str(tmp_path / "output.ply"))
    assert props == ["x", "y", "z"]
    assert np.array_equal(F, tris)
    g = capi.GridMeshCuda(xyz, tris)
    g.GetNeighborsFromTriangles(40)
    capi.EGT_CUDA(g).PerformSmoothing(5, 0.63, -0.64, 1e-8)
    x, y, z = capi.getOutputPoints(g)
    assert np.array_equal(V.astype(np.float32), np.stack([x, y, z], 1))
