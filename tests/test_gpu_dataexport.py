"""Device-side data export: VTKOutput.write downloads the added functions (P1 and P2, FP64 and FP32)
into the files the host writer produces, and checkpoints restore every stored level bit for bit, with
the reference importer's refusals (unknown name, level range, value type, another mesh)."""

import numpy as np
import pytest

import hyteg_b200 as H
from tests.test_dataexport import read_vtu, tet_size

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = H.Context(0)
    yield c
    c.synchronize()


def test_vtk_output_writes_downloaded_functions(ctx, tmp_path):
    pm = H.PrimitiveStorage.cuboid(ctx=ctx)
    nC = pm.counts()[3]
    L = 2
    u = H.P1Function("u", pm, 0, L, ctx)
    f = H.P1Function("f32", pm, 0, L, ctx, dtype="float32")
    q = H.P2Function("q", pm, 0, L, ctx)
    u.fill_random(L, 1)
    f.fill_random(L, 2)
    q.fill_random(L, 3)
    out = H.VTKOutput(str(tmp_path), "sol", pm, writeFrequency=2)
    for fn in (u, f, q):
        out.add(fn)
    out.write(L, 1)  # not a multiple of the frequency: nothing written
    assert not list(tmp_path.iterdir())
    out.setParameter("vtkDataFormat", "BINARY")
    out.write(L, 4)
    p1 = tmp_path / f"sol_VertexDoF_level{L}_ts4.vtu"
    p2 = tmp_path / f"sol_P2_level{L}_ts4.vtu"
    assert p1.exists() and p2.exists()
    n1, c1, _, _, d1 = read_vtu(str(p1))
    n2, c2, _, cells2, d2 = read_vtu(str(p2))
    assert n1 == nC * tet_size((1 << L) + 1) and c1 == nC * 8 ** L
    assert n2 == nC * tet_size((2 << L) + 1) and c2 == nC * 8 ** L and np.all(cells2["types"] == 24)
    for fn, data, Ls in ((u, d1, L), (f, d1, L), (q, d2, L + 1)):
        vals = fn.download(L)
        off, _ = pm.primitive_offsets(Ls)
        ppc = tet_size((1 << Ls) + 1)
        want = np.concatenate([vals[o:o + ppc] for o in off[len(off) - nC:]])
        got = data[fn.name]
        assert np.array_equal(got.astype(np.float64), want.astype(got.dtype).astype(np.float64)), fn.name
    out.remove(f)
    out.setParameter("vtkDataFormat", "ASCII")
    out.write(L, 6)
    _, _, _, _, d = read_vtu(str(tmp_path / f"sol_VertexDoF_level{L}_ts6.vtu"))
    assert set(d) == {"u"}
    assert np.array_equal(d["u"], read_vtu(str(p1))[4]["u"])
    out.close()


def test_checkpoint_round_trip_and_refusals(ctx, tmp_path):
    pm = H.PrimitiveStorage.cuboid(ctx=ctx)
    u = H.P1Function("u", pm, 0, 3, ctx)
    w = H.P2Function("w", pm, 1, 2, ctx, dtype="float32")
    for lv in range(0, 4):
        u.fill_random(lv, 10 + lv)
    for lv in range(1, 3):
        w.fill_random(lv, 20 + lv)
    ex = H.CheckpointExporter()
    ex.registerFunction(u, 1, 3)
    ex.registerFunction(w)
    ex.storeCheckpoint(str(tmp_path), "ck")
    imp = H.CheckpointImporter(str(tmp_path), "ck")
    det = imp.getFunctionDetails()
    assert det == [{"name": "u", "kind": "P1Function", "valueType": "double", "minLevel": 1, "maxLevel": 3},
                   {"name": "w", "kind": "P2Function", "valueType": "float", "minLevel": 1, "maxLevel": 2}]
    u2 = H.P1Function("u", pm, 0, 3, ctx)
    w2 = H.P2Function("w", pm, 1, 2, ctx, dtype="float32")
    imp.restoreFunction(u2, 1, 3)
    imp.restoreFunction(w2)
    for lv in range(1, 4):
        assert np.array_equal(u2.download(lv), u.download(lv))
    for lv in range(1, 3):
        assert np.array_equal(w2.download(lv), w.download(lv))
    with pytest.raises(H.HybError):  # level 0 was not stored
        imp.restoreFunction(u2, 0, 3)
    with pytest.raises(H.HybError):  # stored as double
        imp.restoreFunction(H.P1Function("u", pm, 1, 3, ctx, dtype="float32"), 1, 3)
    with pytest.raises(H.HybError):  # stored as a P2 function
        imp.restoreFunction(H.P1Function("w", pm, 1, 2, ctx, dtype="float32"), 1, 2)
    with pytest.raises(H.HybError):  # not in the checkpoint
        imp.restoreFunction(H.P1Function("z", pm, 1, 3, ctx), 1, 3)
    other = H.PrimitiveStorage.cuboid(nx=2, ctx=ctx)
    with pytest.raises(H.HybError):  # another mesh
        imp.restoreFunction(H.P1Function("u", other, 1, 3, ctx), 1, 3)
