"""GPU parity tests of the elementwise P1 -div(k grad u) operator (p1_div_k_grad_blending_q3) with and
without icosahedral-shell blending, against the oracle assembled from the same element integrals.
Tolerances: apply within 1e-12 relative (max norm over owned DoFs), V-cycle factors within 1e-6."""

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O
from tests import meshes as M

pytestmark = pytest.mark.gpu

K_SPEC = ("expsin", 0.5, (0.13, 0.27, 0.41))
FLAG = O.INNER | O.NEUMANN | O.FREESLIP


def _setup(ctx, mesh, minL, maxL, blending):
    coords, tets = mesh
    om = O.MacroMesh(coords, tets)
    op = O.P1DivKGrad(om, minL, maxL, O.k_expsin(K_SPEC[1], K_SPEC[2]), blending=blending)
    pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
    A = H.P1ElementwiseBlendingDivKGradOperator(pm, minL, maxL, ctx, k=K_SPEC, blending=blending)
    return om, op, pm, A


def _rand(lev, seed, flag=O.ALL):
    rng = np.random.default_rng(seed)
    x = np.zeros(lev.size)
    m = lev.owned_mask(flag)
    x[m] = rng.uniform(-1, 1, m.sum())
    return lev.sync(x)


def _relerr(a, b, mask):
    return np.abs(a[mask] - b[mask]).max() / np.abs(b[mask]).max()


@pytest.mark.parametrize("case", ["cube", "shell"])
@pytest.mark.parametrize("L", [2, 3])
def test_divkgrad_apply_matches_oracle(ctx, case, L):
    mesh = M.cube_6() if case == "cube" else O.mesh_spherical_shell(3, 3, 0.55, 1.0)
    om, op, pm, A = _setup(ctx, mesh, L, L, "shell" if case == "shell" else None)
    lev = op.levels[L]
    x, y0 = _rand(lev, 1), _rand(lev, 2)
    fx = H.P1Function("x", pm, L, L, ctx)
    fy = H.P1Function("y", pm, L, L, ctx)
    fx.upload(L, x)
    fy.upload(L, y0)
    for flag in (O.INNER, O.ALL):
        A.apply(fx, fy, L, flag)
        ref = op.apply(x, y0.copy(), L, flag)
        got = fy.download(L)
        assert _relerr(got, ref, lev.owned_mask(O.ALL)) < 1e-12
        d, s = lev.copy_map()
        np.testing.assert_array_equal(got[d], got[s])
        fy.upload(L, y0)
    # inverse diagonal (computeInverseDiagonalOperatorValues)
    fd = H.P1Function("d", pm, L, L, ctx)
    A.getInverseDiagonalValues(fd, L)
    assert _relerr(fd.download(L), op.invdiag[L], lev.owned_mask(O.ALL)) < 1e-12


def test_divkgrad_smooth_jac(ctx):
    L = 3
    om, op, pm, A = _setup(ctx, M.cube_6(), L, L, None)
    lev = op.levels[L]
    x, b, d0 = _rand(lev, 3), _rand(lev, 4), _rand(lev, 5)
    fx, fb, fd = (H.P1Function(n, pm, L, L, ctx) for n in "xbd")
    fx.upload(L, x)
    fb.upload(L, b)
    fd.upload(L, d0)
    A.smooth_jac(fd, fb, fx, 0.6, L, FLAG)
    ref = op.smooth_jac(d0.copy(), b, x, 0.6, L, FLAG)
    assert _relerr(fd.download(L), ref, lev.owned_mask(O.ALL)) < 1e-12


def test_divkgrad_shell_vcycle_factors(ctx):
    """Configuration-2 shape on a small shell: variable k, shell blending, Chebyshev(3) V(3,3), CG coarse."""
    L = 3
    om, op, pm, A = _setup(ctx, O.mesh_spherical_shell(3, 3, 0.55, 1.0), 0, L, "shell")
    tr = O.Transfer(op)
    lev = op.levels[L]
    b = _rand(lev, 9, O.INNER)
    radii = {l: 2.0 + 0.1 * l for l in range(L + 1)}
    xs = {l: np.zeros(op.levels[l].size) for l in range(L + 1)}
    bs = {l: np.zeros(op.levels[l].size) for l in range(L + 1)}
    bs[L] = b.copy()
    g = O.GMG(op, tr, 0, L, pre=3, post=3, smoother="chebyshev", cheb_order=3, cheb_radii=radii)
    ref = [O.residual_norm(op, xs[L], bs[L], L)]
    for _ in range(4):
        g.solve(xs, bs, L)
        ref.append(O.residual_norm(op, xs[L], bs[L], L))
    ref = np.array(ref)
    fx = H.P1Function("x", pm, 0, L, ctx)
    fb = H.P1Function("b", pm, 0, L, ctx)
    fb.upload(L, b)
    gmg = H.GeometricMultigridSolver(ctx, A, 0, L, preSmoothSteps=3, postSmoothSteps=3, smoother="chebyshev",
                                     chebyshev_order=3)
    gmg.set_radii([radii[l] for l in range(L + 1)])
    hist = gmg.solve_cycles(fx, fb, L, 4)
    np.testing.assert_allclose(hist[0], ref[0], rtol=1e-12)
    np.testing.assert_allclose(hist[1:] / hist[:-1], ref[1:] / ref[:-1], rtol=0, atol=1e-6)
    assert hist[-1] / hist[0] < 1e-2


@pytest.mark.parametrize("case", ["cube", "shell"])
@pytest.mark.parametrize("dtype,tol", [("float64", 1e-13), ("float32", 2e-6)])
def test_divkgrad_stored_element_matrices(ctx, case, dtype, tol):
    """computeAndStoreLocalElementMatrices: applies and smoother sweeps use the stored matrices (kept
    assembled as per-DoF stencils, summed in double) and agree with the recomputing FP64 operator on
    the same stored input values: FP64 within 1e-13 (summation order only), FP32 within its rounding
    of weights, input and result."""
    L = 4
    mesh = M.cube_6() if case == "cube" else O.mesh_spherical_shell(3, 2, 0.55, 1.0)
    bl = "shell" if case == "shell" else None
    coords, tets = mesh
    pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
    A = H.P1ElementwiseBlendingDivKGradOperator(pm, L, L, ctx, k=K_SPEC, blending=bl)
    S = H.P1ElementwiseBlendingDivKGradOperator(pm, L, L, ctx, k=K_SPEC, blending=bl)
    S.computeAndStoreLocalElementMatrices()
    fx, fb = H.P1Function("x", pm, L, L, ctx, dtype), H.P1Function("b", pm, L, L, ctx, dtype)
    fx.fill_random(L, 3)
    fb.fill_random(L, 4)
    # FP64 copies of the stored inputs: the recomputing operator in FP64 is the reference
    gx, gb = H.P1Function("gx", pm, L, L, ctx), H.P1Function("gb", pm, L, L, ctx)
    gx.upload(L, fx.download(L))
    gb.upload(L, fb.download(L))
    ya, ys = H.P1Function("ya", pm, L, L, ctx), H.P1Function("ys", pm, L, L, ctx, dtype)
    for flag in (H.Inner, H.All):
        A.apply(gx, ya, L, flag)
        S.apply(fx, ys, L, flag)
        a, s = ya.download(L), ys.download(L)
        assert np.abs(a - s).max() <= tol * np.abs(a).max()
    A.smooth_jac(ya, gb, gx, 0.6, L, H.Inner)
    S.smooth_jac(ys, fb, fx, 0.6, L, H.Inner)
    a, s = ya.download(L), ys.download(L)
    assert np.abs(a - s).max() <= tol * np.abs(a).max()
