"""GPU parity of the z-streamed cell sweep (levels >= 5, where the bulk-copy ring kernel runs) for
every fused stencil epilogue, against the oracle.

Tolerances as in test_gpu_p1: FP64 within 1e-12 relative (max norm over owned DoFs), V-cycle
factors within 1e-6, FP32 storage within 1e-5, FP16 storage within 5e-3."""

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O
from tests.test_gpu_p1 import FLAG, Setup, _gmg_history, assert_copies_consistent, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8", "cube_2x1x1"])
@pytest.mark.parametrize("L", [5, 6])
def test_zstream_apply_replace_add(ctx, name, L):
    s = Setup(ctx, name, L, L)
    x, y0 = s.rand(L, 21), s.rand(L, 22)
    fx, fy = s.fn("x"), s.fn("y")
    fx.upload(L, x)
    mask = s.op.levels[L].owned_mask(O.ALL)
    for flag in (O.INNER, O.ALL):
        fy.upload(L, y0)
        s.A.apply(fx, fy, L, flag, H.Replace)
        ref = s.op.apply(x, y0.copy(), L, flag)
        got = fy.download(L)
        assert relerr(got, ref, mask) < 1e-12
        assert_copies_consistent(s, L, got)
        s.A.apply(fx, fy, L, flag, H.Add)
        ref2 = s.op.apply(x, ref.copy(), L, flag, add=True)
        assert relerr(fy.download(L), ref2, mask) < 1e-12


@pytest.mark.parametrize("L", [5, 6])
def test_zstream_smooth_jac(ctx, L):
    s = Setup(ctx, "octahedron_8", L, L)
    x, b, d0 = s.rand(L, 1), s.rand(L, 2), s.rand(L, 3)
    fx, fb, fd = s.fn(), s.fn(), s.fn()
    fx.upload(L, x)
    fb.upload(L, b)
    fd.upload(L, d0)
    s.A.smooth_jac(fd, fb, fx, 0.6, L, FLAG)
    ref = s.op.smooth_jac(d0.copy(), b, x, 0.6, L, FLAG)
    got = fd.download(L)
    assert relerr(got, ref, s.op.levels[L].owned_mask(O.ALL)) < 1e-12
    assert_copies_consistent(s, L, got)


def test_zstream_residual_norm(ctx):
    L = 6
    s = Setup(ctx, "cube_6", L, L)
    x, b = s.rand(L, 5), s.rand(L, 6)
    fx, fb, ft = s.fn(), s.fn(), s.fn()
    fx.upload(L, x)
    fb.upload(L, b)
    got = H.residual_norm(s.A, fx, fb, ft, L)
    ref = O.residual_norm(s.op, x, b, L)
    assert abs(got - ref) <= 1e-12 * ref


def test_zstream_chebyshev_vcycle_factors(ctx):
    """Chebyshev smoothing runs the fused CHEB0 / CHEBI / CHEBL epilogues on levels 5 and 6."""
    L = 6
    s = Setup(ctx, "cube_6", 0, L)
    radii = {l: 2.0 + 0.03 * l for l in range(0, L + 1)}
    ref_hist, ref_x, b = _gmg_history(s, L, "chebyshev", 3, radii=radii, pre=2, post=2, cheb_order=3)
    fx, fb = s.fn(), s.fn()
    fb.upload(L, b)
    gmg = H.GeometricMultigridSolver(ctx, s.A, 0, L, preSmoothSteps=2, postSmoothSteps=2, smoother="chebyshev",
                                     chebyshev_order=3)
    gmg.set_radii([radii[l] for l in range(0, L + 1)])
    hist = gmg.solve_cycles(fx, fb, L, 3)
    np.testing.assert_allclose(hist[1:] / hist[:-1], ref_hist[1:] / ref_hist[:-1], rtol=0, atol=1e-6)
    assert relerr(fx.download(L), ref_x, s.op.levels[L].owned_mask(O.ALL)) < 1e-10


@pytest.mark.parametrize("dtype,tol", [("float32", 1e-5), ("float16", 5e-3)])
def test_zstream_low_precision(ctx, dtype, tol):
    L = 6
    s = Setup(ctx, "cube_6", L, L, dtype=dtype)
    x, b = s.rand(L, 7), s.rand(L, 8)
    fx, fy, fb = s.fn(), s.fn(), s.fn()
    fx.upload(L, x)
    fb.upload(L, b)
    s.A.apply(fx, fy, L, O.INNER)
    xq = fx.download(L)
    mask = s.op.levels[L].owned_mask(O.INNER)
    ref = s.op.apply(xq, np.zeros_like(xq), L, O.INNER)
    assert relerr(fy.download(L), ref, mask) < tol
    s.A.smooth_jac(fy, fb, fx, 0.6, L, O.INNER)
    bq = fb.download(L)
    ref = s.op.smooth_jac(np.zeros_like(xq), bq, xq, 0.6, L, O.INNER)
    assert relerr(fy.download(L), ref, mask) < tol


def test_chebyshev_vcycle_factors_fp32(ctx):
    """FP32 storage: the Chebyshev V-cycle on levels 0-6 (fused CHEB0 / CHEBI / CHEBL sweeps on levels 5
    and 6 in FP32) follows the FP64 oracle's residual reduction within 1e-4 per cycle, and its iterate
    within 1e-5."""
    L = 6
    s = Setup(ctx, "cube_6", 0, L, dtype="float32")
    radii = {l: 2.0 + 0.03 * l for l in range(0, L + 1)}
    ref_hist, ref_x, b = _gmg_history(s, L, "chebyshev", 3, radii=radii, pre=2, post=2, cheb_order=3)
    fx, fb = s.fn(), s.fn()
    fb.upload(L, b)
    gmg = H.GeometricMultigridSolver(ctx, s.A, 0, L, preSmoothSteps=2, postSmoothSteps=2, smoother="chebyshev",
                                     chebyshev_order=3)
    gmg.set_radii([radii[l] for l in range(0, L + 1)])
    hist = gmg.solve_cycles(fx, fb, L, 3)
    np.testing.assert_allclose(hist[1:] / hist[:-1], ref_hist[1:] / ref_hist[:-1], rtol=0, atol=1e-4)
    assert relerr(fx.download(L), ref_x, s.op.levels[L].owned_mask(O.ALL)) < 1e-5
