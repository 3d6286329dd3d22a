"""A compiled C++ caller of the C ABI (tests/cpp/gmg_apply.cpp over include/hyteg_b200.hpp, the adaptor
that keeps the reference's class names) runs an apply and six multigrid cycles on the GPU; its results
are checked against the oracle with the tolerances of test_gpu_p1 (apply 1e-12 relative, FP32 storage
1e-5, per-cycle residual-reduction factors 1e-6)."""

import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import hyteg_oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LEVEL = 4


def _u(P):
    return np.sin(3 * P[..., 0]) * np.cos(2 * P[..., 1]) + P[..., 2] ** 2


def _f(P):
    return np.cos(P[..., 0] + 2 * P[..., 1]) * np.exp(P[..., 2])


def _interpolate(lev, fn, flag):
    """Values of fn at the owned slots of `flag` (copies synced), in the layout of the oracle level."""
    v = np.zeros(lev.size)
    pts = O.tet_points(lev.n + 1)
    for c in range(lev.mesh.nC):
        P = lev.coords(c, pts[:, 0], pts[:, 1], pts[:, 2])
        v[lev.owner(c, pts[:, 0], pts[:, 1], pts[:, 2])] = fn(P)
    out = np.zeros(lev.size)
    m = lev.owned_mask(flag)
    out[m] = v[m]
    return lev.sync(out)


@pytest.fixture(scope="module")
def cpp_run(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    out = tmp_path_factory.mktemp("cpp")
    exe = str(out / "gmg_apply")
    libdir = os.path.join(ROOT, "hyteg_b200")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "gmg_apply.cpp"),
                    "-L", libdir, "-lhyteg_b200", f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    r = subprocess.run([exe, str(out), str(LEVEL)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return out


def test_cpp_apply_matches_oracle(cpp_run):
    coords, tets = O.mesh_cuboid()
    m = O.MacroMesh(coords, tets)
    op = O.P1ConstantLaplace(m, LEVEL, LEVEL)
    lev = op.levels[LEVEL]
    x = _interpolate(lev, _u, O.ALL)
    ref = op.apply(x, np.zeros_like(x), LEVEL, O.INNER)
    mask = lev.owned_mask(O.INNER)
    y = np.fromfile(cpp_run / "y.bin", dtype=np.float64)
    y32 = np.fromfile(cpp_run / "y32.bin", dtype=np.float64)
    x32 = np.fromfile(cpp_run / "x32.bin", dtype=np.float64)
    assert y.size == lev.size  # the packed layout of the reference equals the oracle's level layout
    scale = np.abs(ref[mask]).max()
    assert np.abs(y[mask] - ref[mask]).max() < 1e-12 * scale
    # FP32 storage against the oracle on the stored (rounded) input; on a smooth input A x is a small
    # difference of large terms, so the FP32 accumulation error is bounded by the terms, |A| |x|
    x32 = lev.sync(x32.copy())
    ref32 = op.apply(x32, np.zeros_like(x32), LEVEL, O.INNER)
    terms = abs(op.A[LEVEL]) @ np.abs(x32)
    assert np.abs(y32[mask] - ref32[mask]).max() < 1e-5 * terms[mask].max()


def test_cpp_gmg_factors_match_oracle(cpp_run):
    coords, tets = O.mesh_cuboid()
    m = O.MacroMesh(coords, tets)
    op = O.P1ConstantLaplace(m, 0, LEVEL)
    tr = O.Transfer(op)
    b = {l: np.zeros(op.levels[l].size) for l in range(LEVEL + 1)}
    x = {l: np.zeros(op.levels[l].size) for l in range(LEVEL + 1)}
    b[LEVEL] = _interpolate(op.levels[LEVEL], _f, O.INNER)
    g = O.GMG(op, tr, 0, LEVEL, pre=2, post=2)
    ref = [O.residual_norm(op, x[LEVEL], b[LEVEL], LEVEL)]
    for _ in range(6):
        g.solve(x, b, LEVEL)
        ref.append(O.residual_norm(op, x[LEVEL], b[LEVEL], LEVEL))
    hist = np.loadtxt(cpp_run / "hist.txt")
    ref = np.array(ref)
    np.testing.assert_allclose(hist[0], ref[0], rtol=1e-12)
    np.testing.assert_allclose(hist[1:] / hist[:-1], ref[1:] / ref[:-1], rtol=0, atol=1e-6)


def test_cpp_vtk_output_holds_the_functions(cpp_run):
    """The C++ VTKOutput adaptor wrote the level's file; its point data "y" is the macro-cells' arrays of
    the downloaded apply result."""
    from tests.test_dataexport import read_vtu, tet_size

    npts, ncells, _, _, data = read_vtu(str(cpp_run / f"gmg_VertexDoF_level{LEVEL}_ts0.vtu"))
    coords, tets = O.mesh_cuboid()
    m = O.MacroMesh(coords, tets)
    lev = O.Level(m, LEVEL)
    ppc = tet_size((1 << LEVEL) + 1)
    assert npts == m.nC * ppc and ncells == m.nC * 8 ** LEVEL and set(data) == {"x", "y"}
    y = np.fromfile(cpp_run / "y.bin", dtype=np.float64)
    want = np.concatenate([y[o:o + ppc] for o in lev.off_c])
    assert np.array_equal(data["y"], want)
