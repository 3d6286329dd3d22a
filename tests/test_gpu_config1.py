"""Configuration 1 as stated: 3D Poisson on the unit cube split into six macro-tetrahedra, level 5,
FP64, homogeneous Dirichlet BCs, rhs = P1 mass matrix x interpolated f = 3 pi^2 sin(pi x) sin(pi y)
sin(pi z) (the reference's convention: P1ChebyshevSmootherConvergenceTest.cpp:91-93 interpolates the
rhs on All and applies P1ConstantMassOperator with flag All), zero initial guess, V(2,2) weighted
Jacobi omega = 2/3, CG coarse solve on level 0 to 1e-14, ten cycles.

Checked against the oracle: the rhs within 1e-12 relative, every per-cycle residual-reduction factor
within 1e-6, and the solution after ten cycles within 1e-10 relative.
"""

import math

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O

pytestmark = pytest.mark.gpu

L = 5
CYCLES = 10


def f_rhs(x, y, z):
    return 3.0 * math.pi ** 2 * np.sin(math.pi * x) * np.sin(math.pi * y) * np.sin(math.pi * z)


def slot_coords(lev):
    """Coordinates of every owned slot of an oracle level (cell-array points mapped to their owners)."""
    X = np.zeros((lev.size, 3))
    pts = O.tet_points(lev.n + 1)
    for c in range(lev.mesh.nC):
        own = lev.owner(c, pts[:, 0], pts[:, 1], pts[:, 2])
        X[own] = lev.coords(c, pts[:, 0], pts[:, 1], pts[:, 2])
    return X


def test_config1_cube_level5_jacobi_v22(ctx):
    coords, tets = O.mesh_cuboid()
    om = O.MacroMesh(coords, tets)
    op = O.P1ConstantLaplace(om, 0, L)
    mass = O.P1ConstantLaplace(om, L, L, element=O.p1_mass_element)
    lev = op.levels[L]
    all_mask = lev.owned_mask(O.ALL)
    X = slot_coords(lev)
    f = np.zeros(lev.size)
    f[all_mask] = f_rhs(X[all_mask, 0], X[all_mask, 1], X[all_mask, 2])
    lev.sync(f)
    b_ref = lev.sync(mass.apply(f, np.zeros(lev.size), L, O.ALL))

    g = O.GMG(op, O.Transfer(op), 0, L, pre=2, post=2, smoother="jacobi", omega=2.0 / 3.0, cg_tol=1e-14)
    xs = {l: np.zeros(op.levels[l].size) for l in range(L + 1)}
    bs = {l: np.zeros(op.levels[l].size) for l in range(L + 1)}
    bs[L] = b_ref.copy()
    ref_hist = [O.residual_norm(op, xs[L], bs[L], L)]
    for _ in range(CYCLES):
        g.solve(xs, bs, L)
        ref_hist.append(O.residual_norm(op, xs[L], bs[L], L))
    ref_hist = np.array(ref_hist)

    pm = H.PrimitiveStorage.cuboid(ctx=ctx)
    A = H.P1ConstantLaplaceOperator(pm, 0, L, ctx)
    M = H.P1ConstantMassOperator(pm, L, L, ctx)
    ff = H.P1Function("f", pm, 0, L, ctx)
    fb = H.P1Function("b", pm, 0, L, ctx)
    fx = H.P1Function("x", pm, 0, L, ctx)
    ff.interpolate(f_rhs, L, H.All)
    M.apply(ff, fb, L, H.All, H.Replace)
    b = fb.download(L)
    assert np.abs(b[all_mask] - b_ref[all_mask]).max() < 1e-12 * np.abs(b_ref[all_mask]).max()

    gmg = H.GeometricMultigridSolver(ctx, A, 0, L, preSmoothSteps=2, postSmoothSteps=2, smoother="jacobi",
                                     relax=2.0 / 3.0, coarse_rtol=1e-14)
    hist = gmg.solve_cycles(fx, fb, L, CYCLES)
    assert hist.size == CYCLES + 1
    np.testing.assert_allclose(hist[0], ref_hist[0], rtol=1e-12)
    factors, ref_factors = hist[1:] / hist[:-1], ref_hist[1:] / ref_hist[:-1]
    np.testing.assert_allclose(factors, ref_factors, rtol=0, atol=1e-6)
    x = fx.download(L)
    assert np.abs(x[all_mask] - xs[L][all_mask]).max() < 1e-10 * np.abs(xs[L][all_mask]).max()
    # level 0 of this mesh has no inner DoF, so the cycle's coarse correction comes from level 1 up;
    # the oracle's factors are 0.61-0.67 on this problem
    assert factors.max() < 0.7
