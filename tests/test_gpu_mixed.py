"""GPU tests of the mixed-precision defect correction (FP32/FP16 inner multigrid, FP64 outer residual,
update and coarse solve) against the FP64 oracle solution."""

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O
from tests import meshes as M

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("inner", ["float32", "float16"])
def test_mixed_precision_matches_fp64_solution(ctx, inner):
    L = 4
    coords, tets = M.cube_6()
    om = O.MacroMesh(coords, tets)
    op = O.P1ConstantLaplace(om, 0, L)
    tr = O.Transfer(op)
    lev = op.levels[L]
    rng = np.random.default_rng(31)
    b = np.zeros(lev.size)
    mask = lev.owned_mask(O.INNER)
    b[mask] = rng.uniform(-1, 1, mask.sum())
    # FP64 reference solution from the oracle (V-cycles to 1e-13)
    xs = {l: np.zeros(op.levels[l].size) for l in range(L + 1)}
    bs = {l: np.zeros(op.levels[l].size) for l in range(L + 1)}
    bs[L] = b.copy()
    g = O.GMG(op, tr, 0, L, pre=3, post=3)
    r0 = O.residual_norm(op, xs[L], bs[L], L)
    for _ in range(60):
        g.solve(xs, bs, L)
        if O.residual_norm(op, xs[L], bs[L], L) / r0 < 1e-13:
            break
    xref = xs[L]
    pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
    A = H.P1ConstantLaplaceOperator(pm, 0, L, ctx)
    x = H.P1Function("x", pm, L, L, ctx, "float64")
    fb = H.P1Function("b", pm, L, L, ctx, "float64")
    fb.upload(L, b)
    gmg = H.GeometricMultigridSolver(ctx, A, 0, L, preSmoothSteps=3, postSmoothSteps=3, smoother="chebyshev",
                                     chebyshev_order=3)
    hist = gmg.mixed_solve(A, x, fb, L, inner_dtype=inner, inner_cycles=1, max_outer=80, rtol=1e-10)
    assert hist[-1] / hist[0] < 1e-10
    got = x.download(L)
    err = np.linalg.norm(got[mask] - xref[mask]) / np.linalg.norm(xref[mask])
    assert err < 1e-7, err
    # converges at a steady rate: every outer step reduces the residual
    assert np.all(hist[1:] < hist[:-1])
