"""CPU tests: the oracle against the reference's own kernels (golden vectors and, where built, the
compiled reference library) and against the reference tests' known answers."""

import os

import numpy as np
import pytest

from oracle import hyteg_oracle as O
from oracle import ref as R
from tests import meshes as M

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_p1_kernels.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def test_golden_element_matrix(golden):
    K = O.p1_laplace_element(golden["elem_X"])
    np.testing.assert_allclose(K, golden["elem_A"], rtol=0, atol=1e-14)


def test_golden_cell_apply(golden):
    L = int(golden["apply_level"])
    out = O.cell_stencil_apply(golden["apply_src"], L, golden["apply_stencil"])
    np.testing.assert_allclose(out, golden["apply_dst"], rtol=0, atol=1e-14)


def test_golden_restrict(golden):
    L = int(golden["apply_level"])
    out = O.cell_restrict(golden["restrict_fine"], L - 1, golden["nc14"])
    np.testing.assert_allclose(out, golden["restrict_coarse"], rtol=0, atol=1e-14)


def test_golden_prolongate(golden):
    L = int(golden["apply_level"])
    out = O.cell_prolongate(golden["prolong_coarse"], L - 1, golden["nc14"])
    np.testing.assert_allclose(out, golden["prolong_fine"], rtol=0, atol=1e-14)


def _nc14(m, c):
    return ([len(m.e_cells[e]) for e in m.cell_edges[c]] + [len(m.f_cells[f]) for f in m.cell_faces[c]]
            + [len(m.v_cells[v]) for v in m.cells[c]])


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8", "pyramid_4"])
def test_global_operators_match_per_cell_kernels(name):
    """Global A, R, P of the oracle equal the per-cell kernel steps plus additive communication."""
    coords, tets = M.ALL[name]()
    m = O.MacroMesh(coords, tets)
    L = 3
    op = O.P1ConstantLaplace(m, L - 1, L)
    tr = O.Transfer(op)
    fine, coarse = op.levels[L], op.levels[L - 1]
    rng = np.random.default_rng(7)
    x = np.zeros(fine.size)
    x[fine.owned] = rng.uniform(-1, 1, fine.owned.size)
    fine.sync(x)
    fpts, cpts = O.tet_points(fine.n + 1), O.tet_points(coarse.n + 1)
    tot = np.zeros(coarse.size)
    for c in range(m.nC):
        cell = x[fine.off_c[c] + O.cell_index(fine.n, fpts[:, 0], fpts[:, 1], fpts[:, 2])]
        np.add.at(tot, coarse.owner(c, cpts[:, 0], cpts[:, 1], cpts[:, 2]), O.cell_restrict(cell, L - 1, _nc14(m, c)))
    ro = tr.R[L] @ x
    mask = coarse.owned_mask(O.ALL)
    np.testing.assert_allclose(tot[mask], ro[mask], rtol=1e-13, atol=1e-13)
    xc = np.zeros(coarse.size)
    xc[coarse.owned] = rng.uniform(-1, 1, coarse.owned.size)
    coarse.sync(xc)
    tot = np.zeros(fine.size)
    for c in range(m.nC):
        cc = xc[coarse.off_c[c] + O.cell_index(coarse.n, cpts[:, 0], cpts[:, 1], cpts[:, 2])]
        np.add.at(tot, fine.owner(c, fpts[:, 0], fpts[:, 1], fpts[:, 2]), O.cell_prolongate(cc, L - 1, _nc14(m, c)))
    po = tr.P[L] @ xc
    mask = fine.owned_mask(O.ALL)
    np.testing.assert_allclose(tot[mask], po[mask], rtol=1e-13, atol=1e-13)


@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")
def test_assembled_apply_matches_reference_cell_kernel():
    coords, tets = M.cube_6()
    m = O.MacroMesh(coords, tets)
    L = 4
    op = O.P1ConstantLaplace(m, L, L)
    lev = op.levels[L]
    rng = np.random.default_rng(3)
    x = np.zeros(lev.size)
    x[lev.owned] = rng.uniform(-1, 1, lev.owned.size)
    lev.sync(x)
    y = op.A[L] @ x
    pts = O.tet_points(lev.n + 1)
    inner = (pts.min(axis=1) >= 1) & (pts.sum(axis=1) <= lev.n - 1)
    for c in range(m.nC):
        cell = x[lev.off_c[c] + O.cell_index(lev.n, pts[:, 0], pts[:, 1], pts[:, 2])]
        p = lev.owner(c, np.array([2]), np.array([2]), np.array([2]))[0]
        st = [op.A[L][p, lev.owner(c, np.array([2 + d[0]]), np.array([2 + d[1]]), np.array([2 + d[2]]))[0]]
              for d in O.STENCIL15]
        out = R.cell_apply(cell, L, st)
        slots = lev.off_c[c] + O.cell_index(lev.n, pts[inner, 0], pts[inner, 1], pts[inner, 2])
        np.testing.assert_allclose(out[inner], y[slots], rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("name", sorted(M.ALL))
@pytest.mark.parametrize("L", [2, 3])
def test_laplace_annihilates_linear_functions(name, L):
    """P1LaplaceOperator3DTest.cpp:41-127: A u = 0 for constant and linear u at inner DoFs (L2 < 2.8e-13)."""
    coords, tets = M.ALL[name]()
    m = O.MacroMesh(coords, tets)
    op = O.P1ConstantLaplace(m, L, L)
    lev = op.levels[L]
    pts = O.tet_points(lev.n + 1)
    for f in (lambda X: np.ones(len(X)), lambda X: 1.0 + 2 * X[:, 0] - 3 * X[:, 1] + 0.5 * X[:, 2]):
        x = np.zeros(lev.size)
        for c in range(m.nC):
            x[lev.owner(c, pts[:, 0], pts[:, 1], pts[:, 2])] = f(lev.coords(c, pts[:, 0], pts[:, 1], pts[:, 2]))
        y = np.zeros(lev.size)
        op.apply(x, y, L, O.INNER)
        mask = lev.owned_mask(O.INNER)
        if mask.sum() == 0:
            continue
        assert np.sqrt(np.mean(y[mask] ** 2)) < 2.8e-13


def test_restriction_is_prolongation_transpose():
    coords, tets = M.octahedron_8()
    m = O.MacroMesh(coords, tets)
    op = O.P1ConstantLaplace(m, 2, 3)
    tr = O.Transfer(op)
    fi = np.flatnonzero(op.levels[3].owned_mask(O.ALL))
    ci = np.flatnonzero(op.levels[2].owned_mask(O.ALL))
    D = (tr.R[3] - tr.P[3].T).tocsr()[ci][:, fi]
    assert abs(D).max() < 1e-15


def test_chebyshev_polynomial_property():
    """setupCoefficientsInternal: 1 - t p(t) = T_k((theta - t)/delta) / T_k(theta/delta)."""
    for order in range(1, 6):
        lo, hi = 0.3 * 2.2, 1.2 * 2.2
        c = O.chebyshev_coefficients(order, lo, hi)
        theta, delta = (hi + lo) / 2, (hi - lo) / 2
        for t in np.linspace(0.1, 3.0, 7):
            p = sum(ci * t ** i for i, ci in enumerate(c))
            ref = np.polynomial.chebyshev.chebval((theta - t) / delta, [0] * order + [1]) / \
                np.polynomial.chebyshev.chebval(theta / delta, [0] * order + [1])
            assert abs((1 - t * p) - ref) < 1e-12


def test_gmg_convergence_octahedron():
    """P1GMG3DConvergenceTest shape check (there with Gauss-Seidel, bound 3.2e-2 per cycle): weighted-Jacobi
    V(3,3) cycles converge at a rate below 0.2 per cycle on the octahedron."""
    coords, tets = M.octahedron_8()
    m = O.MacroMesh(coords, tets)
    L = 3
    op = O.P1ConstantLaplace(m, 0, L)
    tr = O.Transfer(op)
    rng = np.random.default_rng(0)
    b = {l: np.zeros(op.levels[l].size) for l in range(L + 1)}
    x = {l: np.zeros(op.levels[l].size) for l in range(L + 1)}
    mask = op.levels[L].owned_mask(O.INNER)
    b[L][mask] = rng.uniform(-1, 1, mask.sum())
    g = O.GMG(op, tr, 0, L, pre=3, post=3)
    r0 = O.residual_norm(op, x[L], b[L], L)
    for _ in range(5):
        g.solve(x, b, L)
    r = O.residual_norm(op, x[L], b[L], L)
    assert r / r0 < 0.2 ** 5


def test_cg_solves_small_system():
    coords, tets = M.pyramid_4()
    m = O.MacroMesh(coords, tets)
    L = 2
    op = O.P1ConstantLaplace(m, L, L)
    tr = O.Transfer(op) if False else None
    lev = op.levels[L]
    rng = np.random.default_rng(5)
    b = np.zeros(lev.size)
    mask = lev.owned_mask(O.INNER)
    b[mask] = rng.uniform(-1, 1, mask.sum())
    x = np.zeros(lev.size)
    g = O.GMG(op, tr, L, L, cg_tol=1e-12)
    g.cg(x, b, L)
    assert O.residual_norm(op, x, b, L) / np.linalg.norm(b[mask]) < 1e-11


def test_divkgrad_with_unit_coefficient_is_the_laplacian():
    """p1_div_k_grad with k = 1 and no blending reproduces the P1 Laplace operator."""
    coords, tets = M.octahedron_8()
    m = O.MacroMesh(coords, tets)
    lap = O.P1ConstantLaplace(m, 2, 2)
    dk = O.P1DivKGrad(m, 2, 2, lambda P: np.ones(P.shape[:-1]))
    own = np.flatnonzero(lap.levels[2].owned_mask(O.ALL))
    D = (lap.A[2] - dk.A[2]).tocsr()[own][:, own]
    assert abs(D).max() < 1e-13


@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("map_kind,a", [(0, 0.0), (1, 0.3)])
def test_divkgrad_element_matches_reference_form(map_kind, a):
    """p1_div_k_grad_blending_q3 compiled from the reference sources, with a test blending map."""
    rng = np.random.default_rng(11)
    X = rng.uniform(0, 1, (5, 4, 3))
    K = O.p1_divkgrad_element(X, O.k_expsin(0.5, (0.1, 0.2, 0.3)), None if map_kind == 0 else O.TestMap(a))
    Kr = np.stack([R.p1_divkgrad_blending_element(x, map_kind, a, 0.5, (0.1, 0.2, 0.3)) for x in X])
    np.testing.assert_allclose(K, Kr, rtol=0, atol=1e-13 * np.abs(Kr).max())


def test_shell_map_derivative_and_vertices():
    coords, tets = O.mesh_spherical_shell(3, 3, 0.55, 1.0)
    m = O.MacroMesh(coords, tets)
    rng = np.random.default_rng(4)
    for c in (0, 17, 123, 300, 479):
        B = O.IcosahedralShellMap(m, c)
        P = m.vcoords[list(m.cells[c])]
        np.testing.assert_allclose(B.F(P), P, atol=1e-15)
        X = P.mean(axis=0)[None] + 0.01 * rng.standard_normal((4, 3))
        D = B.DF(X)
        h = 1e-6
        for j in range(3):
            e = np.zeros(3)
            e[j] = h
            np.testing.assert_allclose(D[:, :, j], (B.F(X + e) - B.F(X - e)) / (2 * h), atol=1e-8)


# ------------------------------------------------------------------------------------------ P2
def test_xg4_rule_is_degree_four():
    """The 11-point rule with weights from the moment equations integrates every monomial of degree
    <= 4 on the reference tetrahedron exactly (to rounding) and has positive weights."""
    import math

    P, w = O.XG4_POINTS, O.XG4_WEIGHTS
    assert (w > 0).all()
    for a in range(5):
        for b in range(5 - a):
            for c in range(5 - a - b):
                exact = math.factorial(a) * math.factorial(b) * math.factorial(c) / math.factorial(a + b + c + 3)
                assert abs((w * P[:, 0] ** a * P[:, 1] ** b * P[:, 2] ** c).sum() - exact) < 1e-15


@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("map_kind,a", [(0, 0.0), (1, 0.3)])
def test_p2_divkgrad_element_matches_reference_form(map_kind, a):
    """p2_div_k_grad_blending_q4 compiled from the reference sources, with a test blending map."""
    rng = np.random.default_rng(12)
    X = rng.uniform(0, 1, (5, 4, 3))
    ph = (0.31, 0.12, 0.77)
    K = O.p2_divkgrad_element(X, O.k_expsin(0.5, ph), None if map_kind == 0 else O.TestMap(a))
    Kr = np.stack([R.p2_divkgrad_blending_element(x, map_kind, a, 0.5, ph) for x in X])
    np.testing.assert_allclose(K, Kr, rtol=0, atol=1e-13 * np.abs(Kr).max())


def _slot_coords(lev):
    X = np.full((lev.size, 3), np.nan)
    pts = O.tet_points(lev.n + 1)
    for c in range(lev.mesh.nC):
        X[lev.owner(c, pts[:, 0], pts[:, 1], pts[:, 2])] = lev.coords(c, pts[:, 0], pts[:, 1], pts[:, 2])
    return X


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8", "tilted_tet"])
def test_p2_operator_and_transfer_properties(name):
    """P2 on the node set of level L+1: linear functions are annihilated on inner DoFs, quadratic
    prolongation reproduces quadratics, and (k = 1, affine) A_{L-1} = P^T A_L P (Galerkin)."""
    coords, tets = M.ALL[name]()
    op = O.P2DivKGrad(O.MacroMesh(coords, tets), 1, 3, lambda P: np.ones(len(P)))
    for L in (1, 2, 3):
        lev = op.levels[L]
        X = _slot_coords(lev)
        u = lev.sync(np.nan_to_num(1.0 + 2 * X[:, 0] - 0.5 * X[:, 1] + 0.25 * X[:, 2]))
        assert np.abs((op.A[L] @ u)[lev.owned_mask(O.INNER)]).max() < 1e-13
    for L in (2, 3):
        Pm = O.p2_prolongation_matrix(op.levels[L - 1], op.levels[L])
        Xc, Xf = _slot_coords(op.levels[L - 1]), _slot_coords(op.levels[L])
        q = lambda X: 1 + X[:, 0] ** 2 - 2 * X[:, 1] * X[:, 2] + 0.5 * X[:, 2] + X[:, 0] * X[:, 1]
        uf = Pm @ op.levels[L - 1].sync(np.nan_to_num(q(Xc)))
        ownf = op.levels[L].owned_mask(O.ALL)
        assert np.abs(uf[ownf] - q(Xf)[ownf]).max() < 1e-13
        ownc = op.levels[L - 1].owned_mask(O.ALL)
        Ac = op.A[L - 1][ownc][:, ownc]
        Pf = Pm[ownf][:, ownc]
        assert abs(Pf.T @ op.A[L][ownf][:, ownf] @ Pf - Ac).max() < 1e-13 * abs(Ac).max()


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8", "tilted_tet"])
def test_p2_reference_layout_covers_every_node(name):
    """The reference's P2 memory of level L (vertex-DoF arrays + edge-DoF arrays) addresses exactly
    the nodes of level L+1: every non-ghost entry is a node, and every node has an entry."""
    coords, tets = M.ALL[name]()
    mesh = O.MacroMesh(coords, tets)
    for L in (0, 1, 2):
        X = O.p2_reference_dof_coords(mesh, L)
        lev1 = O.Level(mesh, L + 1)
        nodes = _slot_coords(lev1)[lev1.owned_mask(O.ALL)]
        key = lambda A: {tuple(r) for r in np.round(A, 12)}
        assert key(X[~np.isnan(X[:, 0])]) == key(nodes)
        assert len(key(nodes)) == len(nodes)


def test_p2_reference_edgedof_sizes_example():
    """The layout example of edgedof::macroface::index (EdgeDoFIndexing.hpp:598-611): at level 2 a
    face with one neighbour cell holds 30 own entries and 54 ghost entries."""
    coords, tets = M.ALL["tilted_tet"]()
    mesh = O.MacroMesh(coords, tets)
    sizes = O.edgedof_memory_sizes(mesh, 2)
    assert sizes[mesh.nV + mesh.nE: mesh.nV + mesh.nE + mesh.nF] == [84] * mesh.nF
    assert sizes[-1] == 6 * 20 + 10  # cell: 6 tet(4) + tet(3)
    assert sizes[mesh.nV] == 4 + 2 * 11 + 1 * 21  # edge of one cell, two faces: n + nf(3n-1) + nc(7n-7)


def _ref_lib():
    import ctypes as C
    import os
    p = os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref", "libhyteg_ref.so")
    if not os.path.exists(p):
        pytest.skip("oracle/_ref not built")
    return C.CDLL(p)


@pytest.mark.parametrize("kind,a", [(0, 0.0), (1, 0.3)])
def test_stokes_div_element_matches_reference_forms(kind, a):
    """p2_to_p1_div_{0,1,2}_blending_q2 and p1_to_p2_divt_{0,1,2}_blending_q2 (compiled from the
    reference) equal the oracle's B_k and its transpose; identity and a non-affine test map."""
    import ctypes as C
    lib = _ref_lib()
    X = np.array([[0.1, 0.0, 0.05], [1.0, 0.1, 0.0], [0.2, 0.9, 0.1], [0.05, 0.1, 1.1]])
    B = O.p2p1_div_element(X[None], O.TestMap(a) if kind == 1 else None)[0]
    for k in range(3):
        out = np.zeros(40)
        lib.ref_p2p1_div_element(X.ctypes.data_as(C.c_void_p), kind, C.c_double(a), k, out.ctypes.data_as(C.c_void_p))
        assert np.abs(B[k] - out.reshape(4, 10)).max() < 1e-15
        lib.ref_p1p2_divt_element(X.ctypes.data_as(C.c_void_p), kind, C.c_double(a), k, out.ctypes.data_as(C.c_void_p))
        assert np.abs(B[k].T - out.reshape(10, 4)).max() < 1e-15


@pytest.mark.parametrize("kind,a", [(0, 0.0), (1, 0.3)])
def test_full_viscous_element_matches_reference_forms(kind, a):
    """The nine blocks p2_full_stokesvar_{i}_{j}_blending_q3 (compiled from the reference) equal the
    oracle's full viscous element matrix, with the exp-sin viscosity; identity and a non-affine
    test map, several element shapes."""
    import ctypes as C
    lib = _ref_lib()
    rng = np.random.default_rng(21)
    ph = np.array([0.13, 0.27, 0.41])
    for _ in range(4):
        X = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float) * 0.3 + rng.uniform(-0.05, 0.05, (4, 3)) + 0.2
        K = O.p2_full_viscous_element(X[None], O.k_expsin(0.5, ph), O.TestMap(a) if kind == 1 else None)[0]
        for i in range(3):
            for j in range(3):
                out = np.zeros(100)
                lib.ref_p2_full_viscous_element(X.ctypes.data_as(C.c_void_p), kind, C.c_double(a), i, j, C.c_double(0.5),
                                                ph.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p))
                assert np.abs(K[i, j] - out.reshape(10, 10)).max() <= 1e-13 * np.abs(out).max()


def test_full_viscous_oracle_properties():
    """Rigid-body motions (constant and rotational velocities) are in the kernel of the full viscous
    block on inner DoFs, the operator is symmetric, and its diagonal blocks differ from the
    component Laplacian only by the grad-div terms."""
    coords, tets = M.ALL["cube_6"]()
    mesh = O.MacroMesh(coords, tets)
    op = O.P2FullViscous(mesh, 2, 2, lambda P: np.ones(len(P)))
    L = 2
    lev = op.levels[L]
    X = _slot_coords(lev)
    inner = lev.owned_mask(O.INNER)
    for u in ([np.ones(lev.size), np.zeros(lev.size), np.zeros(lev.size)],
              [-X[:, 1], X[:, 0], np.zeros(lev.size)],
              [np.zeros(lev.size), -X[:, 2], X[:, 1]]):
        y = op.apply(u, [np.zeros(lev.size) for _ in range(3)], L, O.INNER)
        for i in range(3):
            assert np.abs(y[i][inner]).max() < 1e-11
    for i in range(3):
        for j in range(3):
            assert abs(op.A[L][i][j] - op.A[L][j][i].T).max() < 1e-14


def test_pspg_element_matches_reference_form():
    import ctypes as C
    lib = _ref_lib()
    rng = np.random.default_rng(3)
    for _ in range(5):
        X = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float) + 0.2 * rng.uniform(-1, 1, (4, 3))
        out = np.zeros(16)
        lib.ref_p1_pspg_element(X.ravel().ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p))
        K = O.p1_pspg_element(X[None])[0]
        assert np.abs(K - out.reshape(4, 4)).max() < 1e-15 * max(1.0, np.abs(out).max()) * 10


def test_stokes_oracle_vcycle_converges():
    """The Uzawa multigrid restatement converges on the unit cube (eta = 1) with the default
    parameters (the product's defaults)."""
    coords, tets = M.cube_6()
    S = O.P2P1Stokes(O.MacroMesh(coords, tets), 0, 2, lambda P: np.ones(len(P)))
    radii = {l: O.power_iteration_radius(S.Aop, l, np.random.default_rng(40 + l).uniform(-1, 1, S.ulev[l].size), 20)
             for l in range(3)}
    rng = np.random.default_rng(7)
    bu = []
    for _ in range(3):
        x = np.zeros(S.ulev[2].size)
        m = S.umask(2)
        x[m] = rng.uniform(-1, 1, m.sum())
        bu.append(S.ulev[2].sync(x))
    bp = np.zeros(S.plev[2].size)
    u, p = [np.zeros(S.ulev[2].size) for _ in range(3)], np.zeros(S.plev[2].size)
    r = [S.residual_norm(u, p, bu, bp, 2)]
    for _ in range(3):
        u, p = S.vcycle(u, p, bu, bp, 2, radii)
        r.append(S.residual_norm(u, p, bu, bp, 2))
    assert r[-1] < 0.2 * r[0]


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8"])
def test_sor_color_sets(name):
    """The Gauss-Seidel colour sets cover every owned DoF exactly once, the cell-interior colours are a
    proper colouring of the stencil (no coupling inside a set), and a sweep reduces the residual."""
    coords, tets = M.ALL[name]()
    op = O.P1ConstantLaplace(O.MacroMesh(coords, tets), 3, 3)
    L = 3
    lev = op.levels[L]
    sets = O.sor_color_sets(lev)
    owned = np.zeros(lev.size, dtype=bool)
    owned[lev.owned] = True
    count = sum(S.astype(int) for S in sets)
    assert np.all(count[owned] == 1)
    A = op.A[L].tocsr()
    for S in sets[6:]:
        idx = np.flatnonzero(S)
        sub = A[idx][:, idx]
        sub.setdiag(0)
        sub.eliminate_zeros()
        assert sub.nnz == 0
    rng = np.random.default_rng(4)
    x = np.zeros(lev.size)
    m = lev.owned_mask(O.INNER)
    x[m] = rng.uniform(-1, 1, m.sum())
    x = lev.sync(x)
    b = np.zeros(lev.size)
    r0 = np.linalg.norm((b - A @ x)[m])
    y = O.sor_sweep(op, x, b, L, 1.0, O.INNER)
    y = O.sor_sweep(op, y, b, L, 1.0, O.INNER, backwards=True)
    assert np.linalg.norm((b - A @ y)[m]) < 0.8 * r0


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8", "cube_2x1x1", "tilted_tet", "pyramid_4"])
def test_large_level_operator_matches_assembled(name):
    """The large-level oracle (per-cell stencils from element matrices, boundary owners summed over
    their cells' one-sided stencils) equals the assembled operator, here with the reference's own
    compiled cell kernel for the interiors when oracle/_ref is built."""
    coords, tets = M.ALL[name]()
    m = O.MacroMesh(coords, tets)
    L = 3
    op = O.P1ConstantLaplace(m, L, L)
    kernel = R.cell_apply if R.available() else None
    big = O.LargeLevelConstantOperator(m, L, interior_kernel=kernel, level=op.levels[L])
    lev = op.levels[L]
    rng = np.random.default_rng(5)
    x = np.zeros(lev.size)
    x[lev.owned] = rng.uniform(-1, 1, lev.owned.size)
    lev.sync(x)
    mask = lev.owned_mask(O.ALL)
    a = op.apply(x, np.zeros_like(x), L, O.ALL)
    b = big.apply(x, np.zeros_like(x), L, O.ALL)
    assert np.abs(a[mask] - b[mask]).max() <= 1e-14 * np.abs(a[mask]).max()
    np.testing.assert_allclose(big.invdiag[L][mask], op.invdiag[L][mask], rtol=1e-14)
    # like the assembled operator it reads owner slots only: stale copies in the cell arrays (the
    # smoothers' temporaries have them) do not change the result
    x[~lev.owned_mask(O.ALL)] = rng.uniform(-1, 1, (~lev.owned_mask(O.ALL)).sum())
    a = op.apply(x, np.zeros_like(x), L, O.ALL)
    b = big.apply(x, np.zeros_like(x), L, O.ALL)
    assert np.abs(a[mask] - b[mask]).max() <= 1e-14 * np.abs(a[mask]).max()


@pytest.mark.skipif(not R.shell_available(), reason="oracle/_ref shell library not built")
@pytest.mark.parametrize("ntan,nrad", [(3, 2), (5, 3)])
def test_shell_map_matches_reference(ntan, nrad):
    """The oracle's IcosahedralShellMap (vertex classification restated, Jacobian derived
    independently) against the reference's own class, which classifies every macro-cell of the mesh
    itself (skew cells included): F and DF at points inside each cell, to 1e-14 relative."""
    coords, tets = O.mesh_spherical_shell(ntan, nrad, 0.55, 1.0)
    m = O.MacroMesh(coords, tets)
    rng = np.random.default_rng(ntan)
    worst_f = worst_df = 0.0
    for c in range(m.nC):
        P = m.vcoords[list(m.cells[c])]
        lam = rng.dirichlet(np.ones(4), size=5)
        pts = lam @ P
        F, DF, det = R.shell_map_eval(m.vcoords, np.array(m.cells), c, pts)
        mp = O.IcosahedralShellMap(m, c)
        Fo, DFo = mp.F(pts), mp.DF(pts)
        worst_f = max(worst_f, np.abs(Fo - F).max() / np.abs(F).max())
        worst_df = max(worst_df, np.abs(DFo - DF).max() / np.abs(DF).max())
        np.testing.assert_allclose(np.linalg.det(DF), det, rtol=1e-12)
    assert worst_f < 1e-14 and worst_df < 1e-13, (worst_f, worst_df)


def test_p2_nodal_form_reduces_to_the_form_operator_for_constant_k():
    """With a constant coefficient the P2 interpolant is exact, so the nodal-coefficient form equals the
    form-based p2_div_k_grad_blending_q4 operator (blended shell, levels 1 and 2); for the exp-sin
    coefficient the two differ by the interpolation error, which shrinks with the level."""
    coords, tets = O.mesh_spherical_shell(3, 2, 0.55, 1.0)
    om = O.MacroMesh(coords, tets)
    two = lambda P: 2.0 * np.ones(P.shape[:-1])  # noqa: E731
    a = O.P2DivKGrad(om, 1, 1, two, blending="shell")
    b = O.P2DivKGradNodal(om, 1, 1, two, blending="shell")
    d = abs(a.A[1] - b.A[1]).max() / abs(a.A[1]).max()
    assert d < 1e-13
    kfun = O.k_expsin(0.5, (0.13, 0.27, 0.41))
    cube = O.MacroMesh(*O.mesh_cuboid())
    diffs = []
    for L in (1, 2):
        a = O.P2DivKGrad(cube, L, L, kfun)
        b = O.P2DivKGradNodal(cube, L, L, kfun)
        x = np.random.default_rng(L).uniform(-1, 1, a.levels[L].size)
        ya, yb = a.A[L] @ x, b.A[L] @ x
        diffs.append(np.abs(ya - yb).max() / np.abs(ya).max())
    assert diffs[1] < diffs[0]
