"""GPU Gauss-Seidel / SOR of the constant-stencil operator (P1Operator::smooth_sor and GaussSeidelSmoother):
one sweep against the oracle's colour-set sweep (1e-12 relative, forward and backward, relax 1 and
1.3), and the reference's own convergence bound for GMG with Gauss-Seidel smoothing
(tests/hyteg/convergence/P1GMG3DConvergenceTest.cpp: regular octahedron, levels 0-3, V(3,3), CG on
level 0, u = sin(x) sinh(y) z on the boundary, f = 0, random start; the squared discrete residual
must drop by a factor below 3.2e-2 in each of four cycles)."""

import math

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O
from tests.test_gpu_p1 import Setup, assert_copies_consistent, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8", "cube_2x1x1"])
@pytest.mark.parametrize("L", [2, 4])
def test_sor_sweep_matches_oracle(ctx, name, L):
    s = Setup(ctx, name, L, L)
    x, b = s.rand(L, 31), s.rand(L, 32)
    fx, fb = s.fn("x"), s.fn("b")
    fb.upload(L, b)
    mask = s.op.levels[L].owned_mask(O.ALL)
    for relax, backwards in ((1.0, False), (1.3, True)):
        fx.upload(L, x)
        s.A.smooth_sor(fx, fb, relax, L, O.INNER, backwards=backwards)
        ref = O.sor_sweep(s.op, x, b, L, relax, O.INNER, backwards=backwards)
        got = fx.download(L)
        assert relerr(got, ref, mask) < 1e-12, (relax, backwards)
        assert_copies_consistent(s, L, got)


def test_gauss_seidel_multigrid_meets_reference_bound(ctx):
    s = Setup(ctx, "octahedron_8", 0, 3)
    L = 3
    u, f, res, one = s.fn("u"), s.fn("f"), s.fn("r"), s.fn("one")
    one.interpolate(1.0, L)
    u.fill_random(L, 11)
    u.assign([0.5, 0.5], [u, one], L)  # uniform [0, 1] as the reference's start
    u.interpolate(lambda x, y, z: math.sin(x) * math.sinh(y) * z, L, H.DirichletBoundary)
    f.interpolate(0.0, L)
    gmg = H.GeometricMultigridSolver(ctx, s.A, 0, L, 3, 3, smoother="gauss_seidel")
    npts = one.dotGlobal(one, L, H.Inner)
    s.A.apply(u, res, L, H.Inner)
    last = res.dotGlobal(res, L, H.Inner) / npts
    for _ in range(4):
        gmg.solve(s.A, u, f, L)
        s.A.apply(u, res, L, H.Inner)
        cur = res.dotGlobal(res, L, H.Inner) / npts
        assert cur / last < 3.2e-2, cur / last
        last = cur


@pytest.mark.parametrize("dtype,tol", [("float32", 1e-5)])
def test_sor_sweep_low_precision(ctx, dtype, tol):
    L = 4
    s = Setup(ctx, "cube_6", L, L, dtype=dtype)
    x, b = s.rand(L, 41), s.rand(L, 42)
    fx, fb = s.fn("x"), s.fn("b")
    fx.upload(L, x)
    fb.upload(L, b)
    xq, bq = fx.download(L), fb.download(L)
    s.A.smooth_gs(fx, fb, L, O.INNER)
    ref = O.sor_sweep(s.op, xq, bq, L, 1.0, O.INNER)
    assert relerr(fx.download(L), ref, s.op.levels[L].owned_mask(O.ALL)) < tol
