"""CPU tests of the VTK writer (VTKOutput's file layout, dataexport/VTKOutput/VTKOutput.cpp:160-230) on
host data: piece sizes, point positions (affine and under the icosahedral shell map, the latter against
the reference's own IcosahedralShellMap compiled into oracle/_ref), the micro-tetrahedra tiling each
macro-cell, point data equal to the macro-cells' arrays of the packed vector, and binary = ASCII.
The device path (VTKOutput.write, checkpoints) is covered by tests/test_gpu_dataexport.py."""

import base64
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import ref as R


def tet_size(w):
    return (w + 2) * (w + 1) * w // 6


def cidx(n, x, y, z):
    # slice z holds the triangle of side n - z + 1; row y of it starts after the rows below
    w = n + 1
    before = tet_size(w) - tet_size(w - z)
    m = w - z
    return before + (m * (m + 1) // 2 - (m - y) * (m - y + 1) // 2) + x


def read_vtu(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")

    def arr(el):
        types = {"Float64": np.float64, "Float32": np.float32, "Int64": np.int64, "UInt8": np.uint8}
        dt = types[el.get("type")]
        if el.get("format") == "binary":
            raw = base64.b64decode("".join(el.text.split()))
            nbytes = int(np.frombuffer(raw[:4], dtype=np.uint32)[0])
            assert nbytes == len(raw) - 4
            return np.frombuffer(raw[4:], dtype=dt)
        return np.array(el.text.split(), dtype=dt)

    pts = arr(piece.find("Points/DataArray")).reshape(-1, 3)
    cells = {el.get("Name"): arr(el) for el in piece.find("Cells")}
    data = {el.get("Name"): arr(el) for el in piece.find("PointData")}
    return int(piece.get("NumberOfPoints")), int(piece.get("NumberOfCells")), pts, cells, data


def tet_volumes(pts, conn, nv):
    t = conn.reshape(-1, nv)[:, :4]
    a, b, c, d = (pts[t[:, k]] for k in range(4))
    return np.einsum("ij,ij->i", np.cross(b - a, c - a), d - a) / 6.0


def packed_values(pm, Ls, seed):
    return np.random.default_rng(seed).uniform(-1, 1, pm.packed_size(Ls))


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("L", [0, 2])
def test_vtu_cube_layout_geometry_and_data(tmp_path, order, L):
    pm = H.PrimitiveStorage.cuboid()
    nC = pm.counts()[3]
    Ls = L + order - 1
    N = 1 << Ls
    vals = packed_values(pm, Ls, 7)
    path = str(tmp_path / "cube.vtu")
    H.write_vtu_packed(pm, path, L, {"u": vals, "v32": (vals, "float32")}, order=order)
    npts, ncells, pts, cells, data = read_vtu(path)
    assert npts == nC * tet_size(N + 1) and ncells == nC * (1 << L) ** 3
    nv = 10 if order == 2 else 4
    assert np.all(cells["types"] == (24 if order == 2 else 10))
    assert np.array_equal(cells["offsets"], nv * np.arange(1, ncells + 1))
    conn = cells["connectivity"]
    assert conn.min() >= 0 and conn.max() < npts
    # the micro-tetrahedra tile the unit cube: no degenerate cell, volumes sum to one
    vol = np.abs(tet_volumes(pts, conn, nv))
    assert vol.min() > 0 and abs(vol.sum() - 1.0) < 1e-13
    if order == 2:  # edge nodes at the midpoints of the corners
        t = conn.reshape(-1, 10)
        for k, (a, b) in enumerate([(0, 1), (1, 2), (0, 2), (0, 3), (1, 3), (2, 3)]):
            np.testing.assert_allclose(pts[t[:, 4 + k]], 0.5 * (pts[t[:, a]] + pts[t[:, b]]), atol=1e-15)
    # points: each macro-cell's grid in storage order, affine in the cell's vertices
    coords = pm.vertex_coords()
    off, _ = pm.primitive_offsets(Ls)
    cell_off = off[len(off) - nC:]
    ppc = tet_size(N + 1)
    for c in range(nC):
        P = coords[pm.primitive_vertices(3, c)]
        for (x, y, z) in [(0, 0, 0), (N, 0, 0), (0, N, 0), (0, 0, N), (N // 2, 0, N // 2 if N > 1 else 0)]:
            want = P[0] + ((P[1] - P[0]) * x + (P[2] - P[0]) * y + (P[3] - P[0]) * z) / N
            np.testing.assert_allclose(pts[c * ppc + cidx(N, x, y, z)], want, atol=1e-15)
        # point data: the cell's array of the packed vector
        assert np.array_equal(data["u"][c * ppc:(c + 1) * ppc], vals[cell_off[c]:cell_off[c] + ppc])
    assert data["v32"].dtype == np.float32
    np.testing.assert_array_equal(data["v32"], data["u"].astype(np.float32))


def test_vtu_binary_equals_ascii(tmp_path):
    pm = H.PrimitiveStorage.cuboid(nx=2)
    vals = packed_values(pm, 2, 3)
    a, b = str(tmp_path / "a.vtu"), str(tmp_path / "b.vtu")
    H.write_vtu_packed(pm, a, 2, {"u": vals}, binary=False)
    H.write_vtu_packed(pm, b, 2, {"u": vals}, binary=True)
    ra, rb = read_vtu(a), read_vtu(b)
    assert ra[0] == rb[0] and ra[1] == rb[1]
    assert np.array_equal(ra[2], rb[2])
    for k in ra[3]:
        assert np.array_equal(ra[3][k], rb[3][k])
    assert np.array_equal(ra[4]["u"], rb[4]["u"])


@pytest.mark.skipif(not R.shell_available(), reason="oracle/_ref shell library not built")
def test_vtu_p2_shell_nodes_match_reference_map(tmp_path):
    """P2 file on the blended shell: every node of the level+1 grid (vertex and edge nodes of the
    quadratic tetrahedra) is the reference map's image of its affine position, so the edge nodes are
    mapped midpoints, not midpoints of the mapped corners."""
    pm = H.PrimitiveStorage.spherical_shell(3, 2, 0.55, 1.0)
    nC = pm.counts()[3]
    L = 1
    N = 2 << L
    pb, pa = str(tmp_path / "b.vtu"), str(tmp_path / "a.vtu")
    H.write_vtu_packed(pm, pb, L, {}, order=2, blending="shell")
    H.write_vtu_packed(pm, pa, L, {}, order=2)
    _, nc, ptsb, cells, _ = read_vtu(pb)
    _, _, ptsa, _, _ = read_vtu(pa)
    assert nc == nC * 8 ** L and np.all(cells["types"] == 24)
    coords = pm.vertex_coords()
    tets = np.array([pm.primitive_vertices(3, c) for c in range(nC)], dtype=np.int32)
    ppc = tet_size(N + 1)
    for c in range(0, nC, 7):
        F, _, _ = R.shell_map_eval(coords, tets, c, ptsa[c * ppc:(c + 1) * ppc])
        assert np.abs(F - ptsb[c * ppc:(c + 1) * ppc]).max() < 1e-14
    t = cells["connectivity"].reshape(-1, 10)
    mid = 0.5 * (ptsb[t[:, 0]] + ptsb[t[:, 1]])
    assert np.abs(ptsb[t[:, 4]] - mid).max() > 1e-4  # curved edges


@pytest.mark.skipif(not R.shell_available(), reason="oracle/_ref shell library not built")
def test_vtu_shell_points_match_reference_map(tmp_path):
    """Points under the shell blending: every macro-cell's micro-vertices equal the reference's
    IcosahedralShellMap::evalF at their affine positions (1e-14), and the blended micro-tetrahedra fill
    the spherical shell far better than the unblended ones."""
    rmin, rmax = 0.55, 1.0
    pm = H.PrimitiveStorage.spherical_shell(3, 2, rmin, rmax)
    nC = pm.counts()[3]
    L = 2
    N = 1 << L
    path_b, path_a = str(tmp_path / "shell_b.vtu"), str(tmp_path / "shell_a.vtu")
    H.write_vtu_packed(pm, path_b, L, {}, blending="shell", binary=True)
    H.write_vtu_packed(pm, path_a, L, {}, binary=True)
    _, _, pb, cells, _ = read_vtu(path_b)
    _, _, pa, _, _ = read_vtu(path_a)
    coords = pm.vertex_coords()
    tets = np.array([pm.primitive_vertices(3, c) for c in range(nC)], dtype=np.int32)
    ppc = tet_size(N + 1)
    worst = 0.0
    for c in range(nC):
        F, _, _ = R.shell_map_eval(coords, tets, c, pa[c * ppc:(c + 1) * ppc])
        worst = max(worst, np.abs(F - pb[c * ppc:(c + 1) * ppc]).max())
    assert worst < 1e-14, worst
    r = np.linalg.norm(pb, axis=1)
    assert r.min() > rmin - 1e-12 and r.max() < rmax + 1e-12
    exact = 4.0 / 3.0 * np.pi * (rmax ** 3 - rmin ** 3)
    vb = np.abs(tet_volumes(pb, cells["connectivity"], 4)).sum()
    va = np.abs(tet_volumes(pa, cells["connectivity"], 4)).sum()
    assert abs(vb - exact) < 0.25 * abs(va - exact)


def test_vtu_and_checkpoint_arguments_are_checked(tmp_path):
    pm = H.PrimitiveStorage.cuboid()
    with pytest.raises(H.HybError):
        H.write_vtu_packed(pm, str(tmp_path / "x.vtu"), 1, {}, order=3)
    with pytest.raises(H.HybError):
        H.write_vtu_packed(pm, str(tmp_path / "no_such_dir" / "x.vtu"), 1, {})
    w = H.VTKOutput(str(tmp_path), "out", pm)
    with pytest.raises(H.HybError):
        w.setParameter("vtkDataFormat", "XML")
    with pytest.raises(H.HybError):
        w.setParameter("format", "ASCII")
    w.setParameter("vtkDataFormat", "BINARY")
    w.write(1, 0)  # no function added: nothing written
    assert os.listdir(tmp_path) == []
    w.close()
    imp = H.CheckpointImporter(str(tmp_path), "missing")
    with pytest.raises(H.HybError):
        imp.getFunctionDetails()
    bad = tmp_path / "bad.hybckpt"
    bad.write_bytes(b"not a checkpoint at all")
    with pytest.raises(H.HybError):
        H.CheckpointImporter(str(tmp_path), "bad").getFunctionDetails()


def _fake_checkpoint(path, entries, counts=(8, 19, 18, 6), mesh_hash=0):
    """A checkpoint file in the library's format written from Python: magic, version, primitive counts,
    mesh hash, then per function name, kind, value type, level range and per level a packed vector."""
    import struct

    def s(x):
        b = x.encode()
        return struct.pack("<I", len(b)) + b

    out = b"HYBCKPT1" + struct.pack("<I", 1) + struct.pack("<4i", *counts) + struct.pack("<Q", mesh_hash)
    out += struct.pack("<I", len(entries))
    for name, kind, vt, lo, hi in entries:
        out += s(name) + s(kind) + s(vt) + struct.pack("<ii", lo, hi)
        for lv in range(lo, hi + 1):
            n = 3 + lv
            out += struct.pack("<q", n) + np.arange(n, dtype=np.float64).tobytes()
    path.write_bytes(out)


def test_checkpoint_table_is_read_and_checked(tmp_path):
    """getFunctionDetails reads the function table (skipping every level's data); a truncated file and a
    wrong format version are refused."""
    _fake_checkpoint(tmp_path / "ok.hybckpt", [("u", "P1Function", "double", 1, 3), ("w", "P2Function", "float", 0, 2)])
    det = H.CheckpointImporter(str(tmp_path), "ok").getFunctionDetails()
    assert det == [{"name": "u", "kind": "P1Function", "valueType": "double", "minLevel": 1, "maxLevel": 3},
                   {"name": "w", "kind": "P2Function", "valueType": "float", "minLevel": 0, "maxLevel": 2}]
    raw = (tmp_path / "ok.hybckpt").read_bytes()
    (tmp_path / "cut.hybckpt").write_bytes(raw[:60])
    with pytest.raises(H.HybError):
        H.CheckpointImporter(str(tmp_path), "cut").getFunctionDetails()
    (tmp_path / "v2.hybckpt").write_bytes(raw[:8] + (2).to_bytes(4, "little") + raw[12:])
    with pytest.raises(H.HybError):
        H.CheckpointImporter(str(tmp_path), "v2").getFunctionDetails()
