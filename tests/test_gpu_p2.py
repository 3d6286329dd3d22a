"""GPU parity of the P2 path (P2Function, P2 elementwise div-k-grad with and without shell blending,
quadratic transfers, P2 multigrid) against the oracle assembled from the same element integrals
(pinned to the reference's p2_div_k_grad_blending_q4 on the CPU).

Tolerances: apply, smoother and transfers within 1e-12 relative (max norm over owned DoFs), V-cycle
residual-reduction factors within 1e-6."""

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O
from tests import meshes as M

pytestmark = pytest.mark.gpu

K_SPEC = ("expsin", 0.5, (0.13, 0.27, 0.41))
FLAG = O.INNER | O.NEUMANN | O.FREESLIP


def _mesh(case):
    return M.cube_6() if case == "cube" else O.mesh_spherical_shell(3, 2, 0.55, 1.0)


def _setup(ctx, case, minL, maxL):
    coords, tets = _mesh(case)
    om = O.MacroMesh(coords, tets)
    bl = "shell" if case == "shell" else None
    op = O.P2DivKGrad(om, minL, maxL, O.k_expsin(K_SPEC[1], K_SPEC[2]), blending=bl)
    pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
    A = H.P2ElementwiseBlendingDivKGradOperator(pm, minL, maxL, ctx, k=K_SPEC, blending=bl)
    return om, op, pm, A


def _rand(lev, seed, flag=O.ALL):
    rng = np.random.default_rng(seed)
    x = np.zeros(lev.size)
    m = lev.owned_mask(flag)
    x[m] = rng.uniform(-1, 1, m.sum())
    return lev.sync(x)


def _relerr(a, b, mask):
    return np.abs(a[mask] - b[mask]).max() / max(np.abs(b[mask]).max(), 1e-300)


@pytest.mark.parametrize("case", ["cube", "shell"])
@pytest.mark.parametrize("L", [1, 2, 3])
def test_p2_apply_and_diagonal_match_oracle(ctx, case, L):
    om, op, pm, A = _setup(ctx, case, L, L)
    lev = op.levels[L]
    x, y0 = _rand(lev, 1), _rand(lev, 2)
    fx, fy = H.P2Function("x", pm, L, L, ctx), H.P2Function("y", pm, L, L, ctx)
    fx.upload(L, lev_pack(pm, lev, L, x))
    mask = lev.owned_mask(O.ALL)
    for flag in (O.INNER, O.ALL):
        fy.upload(L, lev_pack(pm, lev, L, y0))
        A.apply(fx, fy, L, flag)
        ref = op.apply(x, y0.copy(), L, flag)
        got = lev_unpack(pm, lev, L, fy.download(L))
        assert _relerr(got, ref, mask) < 1e-12
        d, s = lev.copy_map()
        np.testing.assert_array_equal(got[d], got[s])
    fd = H.P2Function("d", pm, L, L, ctx)
    A.getInverseDiagonalValues(fd, L)
    got = lev_unpack(pm, lev, L, fd.download(L))
    own = lev.owned_mask(O.ALL)
    assert _relerr(got, op.invdiag[L], own) < 1e-12


def lev_pack(pm, lev, L, v):
    """oracle slot vector (Level L+1 layout) -> packed level vector of the P2 function"""
    return v[_packed_index(pm, lev, L)]


def lev_unpack(pm, lev, L, packed):
    out = np.zeros(lev.size)
    out[_packed_index(pm, lev, L)] = packed
    return out


def _packed_index(pm, lev, L):
    # packed layout = oracle slot layout without padding; the oracle Level has no padding
    off, sz = pm.primitive_offsets(L + 1)
    assert pm.packed_size(L + 1) == lev.size
    return np.arange(lev.size)


@pytest.mark.parametrize("case", ["cube", "shell"])
def test_p2_smooth_jac_and_stored_matrices(ctx, case):
    L = 2
    om, op, pm, A = _setup(ctx, case, L, L)
    lev = op.levels[L]
    x, b, d0 = _rand(lev, 3), _rand(lev, 4), _rand(lev, 5)
    fx, fb, fd = (H.P2Function(n, pm, L, L, ctx) for n in ("x", "b", "d"))
    fx.upload(L, x)
    fb.upload(L, b)
    fd.upload(L, d0)
    A.smooth_jac(fd, fb, fx, 0.6, L, FLAG)
    ref = op.smooth_jac(d0.copy(), b, x, 0.6, L, FLAG)
    mask = lev.owned_mask(O.ALL)
    assert _relerr(fd.download(L), ref, mask) < 1e-12
    S = H.P2ElementwiseBlendingDivKGradOperator(pm, L, L, ctx, k=K_SPEC, blending="shell" if case == "shell" else None)
    S.computeAndStoreLocalElementMatrices()
    fy = H.P2Function("y", pm, L, L, ctx)
    S.apply(fx, fy, L, O.ALL)
    assert _relerr(fy.download(L), op.apply(x, np.zeros_like(x), L, O.ALL), mask) < 1e-12


@pytest.mark.parametrize("case", ["cube", "shell"])
def test_p2_transfers_match_oracle(ctx, case):
    L = 3
    om, op, pm, A = _setup(ctx, case, L - 1, L)
    tr = O.P2Transfer(op)
    f = H.P2Function("f", pm, L - 1, L, ctx)
    fine, coarse = _rand(op.levels[L], 6), _rand(op.levels[L - 1], 7)
    f.upload(L, fine)
    f.upload(L - 1, coarse)
    H.P2toP2QuadraticRestriction().restrict(f, L, O.ALL)
    ref = tr.restrict(fine, coarse.copy(), L, O.ALL)
    assert _relerr(f.download(L - 1), ref, op.levels[L - 1].owned_mask(O.ALL)) < 1e-12
    f.upload(L - 1, coarse)
    H.P2toP2QuadraticProlongation().prolongateAndAdd(f, L - 1, FLAG)
    ref = tr.prolongate(coarse, fine.copy(), L, FLAG, add=True)
    got = f.download(L)
    assert _relerr(got, ref, op.levels[L].owned_mask(O.ALL)) < 1e-12
    d, s = op.levels[L].copy_map()
    np.testing.assert_array_equal(got[d], got[s])


@pytest.mark.parametrize("case", ["cube", "shell"])
def test_p2_gmg_chebyshev_factors(ctx, case):
    """P2 multigrid (config 2's solver shape on small levels): V(3,3) Chebyshev(3), quadratic transfers,
    CG coarse solve; per-cycle residual reduction factors within 1e-6 of the oracle's."""
    minL, L = 0, 2
    om, op, pm, A = _setup(ctx, case, minL, L)
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


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8"])
@pytest.mark.parametrize("L", [0, 1, 3])
def test_p2_reference_layout_download_upload(ctx, name, L):
    """hyb_p2_fn_download_reference puts every DoF where the reference's P2Function memory keeps it
    (the oracle gives each entry's coordinates), writes ghost entries as zero, and upload_reference
    restores the function bit for bit."""
    coords, tets = M.ALL[name]()
    om = O.MacroMesh(coords, tets)
    pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
    f = lambda x, y, z: 1.0 + 0.5 * x - 2.0 * y * y + 3.0 * x * z + 0.25 * np.sin(3.0 * x + 7.0 * y - 5.0 * z)
    u = H.P2Function("u", pm, L, L, ctx)
    u.interpolate(f, L)
    got = u.download_reference(L)
    X = O.p2_reference_dof_coords(om, L)
    assert got.size == X.shape[0] == sum(u.reference_layout_sizes(L))
    own = ~np.isnan(X[:, 0])
    np.testing.assert_allclose(got[own], f(X[own, 0], X[own, 1], X[own, 2]), rtol=0, atol=1e-14)
    assert not got[~own].any()
    w = H.P2Function("w", pm, L, L, ctx)
    w.upload_reference(L, got)
    lev1 = O.Level(om, L + 1)  # storage: owned slots and their copies in the cell arrays
    keep = lev1.owned_mask(O.ALL)
    keep[lev1.copy_map()[0]] = True
    np.testing.assert_array_equal(w.download(L)[keep], u.download(L)[keep])
    np.testing.assert_array_equal(w.download_reference(L), got)
