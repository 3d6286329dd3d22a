"""GPU parity of the P2 constant-stencil Laplacian (P2ConstantLaplaceOperator, P2ConstantOperator.cpp:
100-114) against the oracle, which assembles the P2 Laplacian from the element matrices of every
micro-cell (the reference form p2_div_k_grad_blending_q4 with k = 1 and no blending; its degree-4 rule
integrates the constant-coefficient P2 stiffness exactly).  On levels too large for the oracle the
stencil sweep is compared with the GPU's elementwise P2 operator with k = 1, itself pinned to the
oracle in tests/test_gpu_p2.py.

Tolerances: apply, smoother, inverse diagonal within 1e-12 relative (max norm over owned DoFs), FP32
storage within 1e-5, V-cycle residual-reduction factors within 1e-6."""

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O
from tests import meshes as M

pytestmark = pytest.mark.gpu

FLAG = O.INNER | O.NEUMANN | O.FREESLIP


def _one(P):
    return np.ones(P.shape[:-1])


def _setup(ctx, name, minL, maxL, dtype="float64"):
    coords, tets = M.ALL[name]()
    om = O.MacroMesh(coords, tets)
    op = O.P2DivKGrad(om, minL, maxL, _one)
    pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
    A = H.P2ConstantLaplaceOperator(pm, minL, maxL, ctx)
    return op, pm, A


def _rand(lev, seed, flag=O.ALL):
    rng = np.random.default_rng(seed)
    x = np.zeros(lev.size)
    m = lev.owned_mask(flag)
    x[m] = rng.uniform(-1, 1, m.sum())
    return lev.sync(x)


def _relerr(a, b, mask):
    return np.abs(a[mask] - b[mask]).max() / max(np.abs(b[mask]).max(), 1e-300)


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8", "pyramid_4", "tilted_tet", "cube_2x1x1"])
@pytest.mark.parametrize("L", [1, 2, 3])
def test_p2_constant_apply_matches_oracle(ctx, name, L):
    op, pm, A = _setup(ctx, name, L, L)
    lev = op.levels[L]
    x, y0 = _rand(lev, 1), _rand(lev, 2)
    fx, fy = H.P2Function("x", pm, L, L, ctx), H.P2Function("y", pm, L, L, ctx)
    fx.upload(L, x)
    mask = lev.owned_mask(O.ALL)
    d, s = lev.copy_map()
    for flag in (O.INNER, O.ALL):
        for update in (H.Replace, H.Add):
            fy.upload(L, y0)
            A.apply(fx, fy, L, flag, update)
            ref = op.apply(x, y0.copy(), L, flag, add=(update == H.Add))
            got = fy.download(L)
            assert _relerr(got, ref, mask) < 1e-12, (flag, update)
            np.testing.assert_array_equal(got[d], got[s])


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8"])
def test_p2_constant_inverse_diagonal_and_jacobi(ctx, name):
    L = 3
    op, pm, A = _setup(ctx, name, L, L)
    lev = op.levels[L]
    fd = H.P2Function("d", pm, L, L, ctx)
    A.getInverseDiagonalValues(fd, L)
    own = lev.owned_mask(O.ALL)
    assert _relerr(fd.download(L), op.invdiag[L], own) < 1e-12
    x, b, d0 = _rand(lev, 3), _rand(lev, 4), _rand(lev, 5)
    fx, fb, fo = (H.P2Function(n, pm, L, L, ctx) for n in ("x", "b", "o"))
    fx.upload(L, x)
    fb.upload(L, b)
    fo.upload(L, d0)
    A.smooth_jac(fo, fb, fx, 0.6, L, FLAG)
    ref = op.smooth_jac(d0.copy(), b, x, 0.6, L, FLAG)
    assert _relerr(fo.download(L), ref, own) < 1e-12


@pytest.mark.parametrize("name,L", [("cube_6", 5), ("cube_6", 6), ("octahedron_8", 5)])
def test_p2_constant_matches_elementwise_on_large_levels(ctx, name, L):
    """Levels whose cell interiors are cut into many sweep units (several 64-point tiles per row and
    several slice ranges per tile column): the stencil sweep against the elementwise operator."""
    coords, tets = M.ALL[name]()
    pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
    A = H.P2ConstantLaplaceOperator(pm, L, L, ctx)
    E = H.P2ElementwiseBlendingDivKGradOperator(pm, L, L, ctx)
    fx, fy, fz = (H.P2Function(n, pm, L, L, ctx) for n in ("x", "y", "z"))
    fx.fill_random(L, 17)
    fy.fill_random(L, 18)
    fz.copyFrom(fy, L)
    for flag in (H.Inner, H.All):
        A.apply(fx, fy, L, flag)
        E.apply(fx, fz, L, flag)
        a, e = fy.download(L), fz.download(L)
        assert np.abs(a - e).max() < 1e-12 * np.abs(e).max(), flag


@pytest.mark.parametrize("dtype,tol", [("float32", 1e-5), ("float16", 5e-3)])
def test_p2_constant_low_precision_storage(ctx, dtype, tol):
    L = 3
    op, pm, A = _setup(ctx, "cube_6", L, L)
    lev = op.levels[L]
    x = _rand(lev, 9)
    fx, fy = H.P2Function("x", pm, L, L, ctx, dtype), H.P2Function("y", pm, L, L, ctx, dtype)
    fx.upload(L, x)
    A.apply(fx, fy, L, O.INNER)
    xs = fx.download(L)  # the stored (rounded) input
    ref = op.apply(xs, np.zeros_like(xs), L, O.INNER)
    mask = lev.owned_mask(O.INNER)
    assert _relerr(fy.download(L), ref, mask) < tol


def test_p2_constant_gmg_chebyshev_factors(ctx):
    """P2 multigrid with the constant operator: V(3,3) Chebyshev(3), quadratic transfers, CG coarse
    solve; per-cycle residual reduction factors within 1e-6 of the oracle's."""
    minL, L = 0, 3
    op, pm, A = _setup(ctx, "cube_6", minL, L)
    tr = O.P2Transfer(op)
    radii = {l: 2.5 + 0.1 * l for l in range(minL, L + 1)}
    lev = op.levels[L]
    b = _rand(lev, 8, O.INNER)
    bs = {l: np.zeros(op.levels[l].size) for l in range(minL, L + 1)}
    xs = {l: np.zeros(op.levels[l].size) for l in range(minL, L + 1)}
    bs[L] = b.copy()
    g = O.GMG(op, tr, minL, L, smoother="chebyshev", cheb_radii=radii, pre=3, post=3, cheb_order=3)
    hist = [O.residual_norm(op, xs[L], bs[L], L)]
    for _ in range(4):
        g.solve(xs, bs, L)
        hist.append(O.residual_norm(op, xs[L], bs[L], L))
    hist = np.array(hist)
    fx, fb = H.P2Function("x", pm, minL, L, ctx), H.P2Function("b", pm, minL, L, ctx)
    fb.upload(L, b)
    gmg = H.GeometricMultigridSolver(ctx, A, minL, L, 3, 3, smoother="chebyshev", chebyshev_order=3)
    gmg.set_radii([radii[l] for l in range(minL, L + 1)])
    got = gmg.solve_cycles(fx, fb, L, 4)
    np.testing.assert_allclose(got[0], hist[0], rtol=1e-12)
    np.testing.assert_allclose(got[1:] / got[:-1], hist[1:] / hist[:-1], rtol=0, atol=1e-6)
    assert _relerr(fx.download(L), xs[L], lev.owned_mask(O.ALL)) < 1e-9


def test_p2_constant_refuses_sor_and_stencil_query(ctx):
    coords, tets = M.cube_6()
    pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
    A = H.P2ConstantLaplaceOperator(pm, 2, 2, ctx)
    fx, fb = H.P2Function("x", pm, 2, 2, ctx), H.P2Function("b", pm, 2, 2, ctx)
    with pytest.raises(H.HybError):
        A.smooth_sor(fx, fb, 1.0, 2, H.Inner)
    with pytest.raises(H.HybError):
        A.stencil(2, 0)
