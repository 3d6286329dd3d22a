"""GPU parity tests: the CUDA path, called through the C ABI, against the oracle.

Tolerances: FP64 apply/transfer/smoother results within 1e-12 relative (max-norm over owned DoFs);
per-cycle multigrid residual-reduction factors within 1e-6; FP32 storage within 1e-5 and FP16
storage within 5e-3 relative of the FP64 oracle.
"""

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O
from tests import meshes as M

pytestmark = pytest.mark.gpu

FLAG = O.INNER | O.NEUMANN | O.FREESLIP


class Setup:
    def __init__(self, ctx, name, minL, maxL, dtype="float64"):
        coords, tets = M.ALL[name]()
        self.om = O.MacroMesh(coords, tets)
        self.op = O.P1ConstantLaplace(self.om, minL, maxL)
        self.tr = O.Transfer(self.op)
        self.pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
        self.A = H.P1ConstantLaplaceOperator(self.pm, minL, maxL, ctx)
        self.ctx, self.minL, self.maxL, self.dtype = ctx, minL, maxL, dtype

    def fn(self, name="f"):
        return H.P1Function(name, self.pm, self.minL, self.maxL, self.ctx, self.dtype)

    def rand(self, L, seed, flag=O.ALL):
        lev = self.op.levels[L]
        rng = np.random.default_rng(seed)
        x = np.zeros(lev.size)
        m = lev.owned_mask(flag)
        x[m] = rng.uniform(-1, 1, m.sum())
        return lev.sync(x)


def relerr(a, b, mask):
    d = np.abs(a[mask] - b[mask]).max()
    s = max(np.abs(b[mask]).max(), 1e-300)
    return d / s


def assert_copies_consistent(s, L, vec):
    d, src = s.op.levels[L].copy_map()
    np.testing.assert_array_equal(vec[d], vec[src])


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8", "pyramid_4", "tilted_tet", "cube_2x1x1"])
@pytest.mark.parametrize("L", [2, 3, 5])
@pytest.mark.parametrize("flag", [O.INNER, O.ALL])
def test_apply_matches_oracle(ctx, name, L, flag):
    s = Setup(ctx, name, L, L)
    x = s.rand(L, 11)
    y0 = s.rand(L, 12)
    fx, fy = s.fn("x"), s.fn("y")
    fx.upload(L, x)
    fy.upload(L, y0)
    s.A.apply(fx, fy, L, flag, H.Replace)
    got = fy.download(L)
    ref = s.op.apply(x, y0.copy(), L, flag)
    lev = s.op.levels[L]
    mask = lev.owned_mask(O.ALL)
    assert relerr(got, ref, mask) < 1e-12
    assert_copies_consistent(s, L, got)
    # Add
    s.A.apply(fx, fy, L, flag, H.Add)
    got2 = fy.download(L)
    ref2 = s.op.apply(x, ref.copy(), L, flag, add=True)
    assert relerr(got2, ref2, mask) < 1e-12


def test_apply_level_edges(ctx):
    """levels 0 and 1: no cell or face interiors; edges and vertices only."""
    s = Setup(ctx, "octahedron_8", 0, 1)
    for L in (0, 1):
        x = s.rand(L, 3)
        fx, fy = s.fn(), s.fn()
        fx.upload(L, x)
        s.A.apply(fx, fy, L, O.ALL)
        ref = s.op.apply(x, np.zeros_like(x), L, O.ALL)
        mask = s.op.levels[L].owned_mask(O.ALL)
        assert relerr(fy.download(L), ref, mask) < 1e-12


def test_smooth_jac_matches_oracle(ctx):
    L = 4
    s = Setup(ctx, "cube_6", L, L)
    x, b, dst0 = s.rand(L, 1), s.rand(L, 2), s.rand(L, 3)
    fx, fb, fd = s.fn(), s.fn(), s.fn()
    fx.upload(L, x)
    fb.upload(L, b)
    fd.upload(L, dst0)
    s.A.smooth_jac(fd, fb, fx, 2.0 / 3.0, L, FLAG)
    ref = s.op.smooth_jac(dst0.copy(), b, x, 2.0 / 3.0, L, FLAG)
    mask = s.op.levels[L].owned_mask(O.ALL)
    got = fd.download(L)
    assert relerr(got, ref, mask) < 1e-12
    assert_copies_consistent(s, L, got)


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8", "cube_2x1x1"])
def test_restrict_prolongate_match_oracle(ctx, name):
    L = 4
    s = Setup(ctx, name, L - 1, L)
    f = s.fn()
    fine = s.rand(L, 5)
    coarse0 = s.rand(L - 1, 6)
    f.upload(L, fine)
    f.upload(L - 1, coarse0)
    H.P1toP1LinearRestriction().restrict(f, L, FLAG)
    got = f.download(L - 1)
    ref = s.tr.restrict(fine, coarse0.copy(), L, FLAG)
    cmask = s.op.levels[L - 1].owned_mask(O.ALL)
    assert relerr(got, ref, cmask) < 1e-12
    assert_copies_consistent(s, L - 1, got)
    # prolongateAndAdd from the restricted coarse values
    H.P1toP1LinearProlongation().prolongateAndAdd(f, L - 1, FLAG)
    gotf = f.download(L)
    reff = s.tr.prolongate(ref, fine.copy(), L, FLAG, add=True)
    fmask = s.op.levels[L].owned_mask(O.ALL)
    assert relerr(gotf, reff, fmask) < 1e-12
    assert_copies_consistent(s, L, gotf)
    # prolongate (Replace)
    H.P1toP1LinearProlongation().prolongate(f, L - 1, FLAG)
    reff2 = s.tr.prolongate(ref, reff.copy(), L, FLAG, add=False)
    assert relerr(f.download(L), reff2, fmask) < 1e-12


def test_blas1_and_dot(ctx):
    L = 4
    s = Setup(ctx, "octahedron_8", L, L)
    a, b, c = s.rand(L, 1), s.rand(L, 2), s.rand(L, 3)
    fa, fb, fc = s.fn(), s.fn(), s.fn()
    fa.upload(L, a)
    fb.upload(L, b)
    fc.upload(L, c)
    lev = s.op.levels[L]
    for flag in (O.INNER, O.ALL, O.DIRICHLET):
        m = lev.owned_mask(flag)
        assert abs(fa.dotGlobal(fb, L, flag) - O.dot(lev, a, b, flag)) < 1e-12 * max(1, abs(O.dot(lev, a, b, flag)))
    fc.assign([2.0, -0.5], [fa, fb], L, O.INNER)
    ref = c.copy()
    m = lev.owned_mask(O.INNER)
    ref[m] = 2.0 * a[m] - 0.5 * b[m]
    got = fc.download(L)
    mall = lev.owned_mask(O.ALL)
    assert relerr(got, ref, mall) < 1e-15
    assert_copies_consistent(s, L, got)
    fc.add([3.0], [fa], L, O.ALL)
    ref[mall] += 3.0 * a[mall]
    assert relerr(fc.download(L), ref, mall) < 1e-14
    fc.interpolate(1.5, L, O.DIRICHLET)
    ref[lev.owned_mask(O.DIRICHLET)] = 1.5
    assert relerr(fc.download(L), ref, mall) < 1e-14
    # deterministic reductions: bitwise equal on repeat
    d1 = fa.dotGlobal(fb, L, O.ALL)
    d2 = fa.dotGlobal(fb, L, O.ALL)
    assert d1 == d2


def test_interpolate_callback_and_inverse_diagonal(ctx):
    L = 3
    s = Setup(ctx, "cube_6", L, L)
    f = s.fn()
    f.interpolate(lambda x, y, z: 1.0 + x - 2 * y + 3 * z, L, O.ALL)
    got = f.download(L)
    lev = s.op.levels[L]
    pts = O.tet_points(lev.n + 1)
    ref = np.zeros(lev.size)
    for c in range(s.om.nC):
        X = lev.coords(c, pts[:, 0], pts[:, 1], pts[:, 2])
        ref[lev.owner(c, pts[:, 0], pts[:, 1], pts[:, 2])] = 1.0 + X[:, 0] - 2 * X[:, 1] + 3 * X[:, 2]
    mask = lev.owned_mask(O.ALL)
    assert relerr(got, ref, mask) < 1e-14
    d = s.fn()
    s.A.getInverseDiagonalValues(d, L, O.ALL)
    assert relerr(d.download(L), s.op.invdiag[L], mask) < 1e-13


def test_cg_matches_oracle(ctx):
    L = 3
    s = Setup(ctx, "octahedron_8", L, L)
    b = s.rand(L, 8, O.INNER)
    fx, fb = s.fn(), s.fn()
    fb.upload(L, b)
    cg = H.CGSolver(s.pm, L, L, maxIter=500, relativeTolerance=1e-12, absoluteTolerance=1e-30)
    cg.solve(s.A, fx, fb, L)
    x = np.zeros_like(b)
    g = O.GMG(s.op, None, L, L, cg_tol=1e-12, cg_abs=1e-30, cg_maxit=500)
    it = g.cg(x, b, L)
    mask = s.op.levels[L].owned_mask(O.ALL)
    assert relerr(fx.download(L), x, mask) < 1e-9
    assert abs(cg.iterations - (it + 1)) <= 1


def _gmg_history(s, L, smoother, cycles, radii=None, **kw):
    rng_b = s.rand(L, 21, O.INNER)
    # oracle
    b = {l: np.zeros(s.op.levels[l].size) for l in range(s.minL, L + 1)}
    x = {l: np.zeros(s.op.levels[l].size) for l in range(s.minL, L + 1)}
    b[L] = rng_b.copy()
    g = O.GMG(s.op, s.tr, s.minL, L, smoother=smoother, cheb_radii=radii, **kw)
    hist = [O.residual_norm(s.op, x[L], b[L], L)]
    for _ in range(cycles):
        g.solve(x, b, L)
        hist.append(O.residual_norm(s.op, x[L], b[L], L))
    return np.array(hist), x[L], rng_b


@pytest.mark.parametrize("use_graph", [False, True])
def test_gmg_jacobi_vcycle_factors(ctx, use_graph):
    """Config-1 style: 6-tet cube, V(2,2) weighted Jacobi 2/3, CG coarse; per-cycle factors within 1e-6."""
    L = 4
    s = Setup(ctx, "cube_6", 0, L)
    ref_hist, ref_x, b = _gmg_history(s, L, "jacobi", 6, pre=2, post=2)
    fx, fb = s.fn(), s.fn()
    fb.upload(L, b)
    gmg = H.GeometricMultigridSolver(ctx, s.A, 0, L, preSmoothSteps=2, postSmoothSteps=2, relax=2.0 / 3.0,
                                     use_graph=use_graph)
    hist = gmg.solve_cycles(fx, fb, L, 6)
    np.testing.assert_allclose(hist[0], ref_hist[0], rtol=1e-12)
    np.testing.assert_allclose(hist[1:] / hist[:-1], ref_hist[1:] / ref_hist[:-1], rtol=0, atol=1e-6)
    mask = s.op.levels[L].owned_mask(O.ALL)
    assert relerr(fx.download(L), ref_x, mask) < 1e-10


def test_gmg_chebyshev_vcycle_factors(ctx):
    L = 4
    s = Setup(ctx, "octahedron_8", 0, L)
    radii = {l: 2.0 + 0.05 * l for l in range(0, L + 1)}
    ref_hist, ref_x, b = _gmg_history(s, L, "chebyshev", 5, radii=radii, pre=3, post=3, cheb_order=3)
    fx, fb = s.fn(), s.fn()
    fb.upload(L, b)
    gmg = H.GeometricMultigridSolver(ctx, s.A, 0, L, preSmoothSteps=3, postSmoothSteps=3, smoother="chebyshev",
                                     chebyshev_order=3)
    gmg.set_radii([radii[l] for l in range(0, L + 1)])
    hist = gmg.solve_cycles(fx, fb, L, 5)
    np.testing.assert_allclose(hist[1:] / hist[:-1], ref_hist[1:] / ref_hist[:-1], rtol=0, atol=1e-6)


def test_power_iteration_radius(ctx):
    L = 3
    s = Setup(ctx, "cube_6", L, L)
    x0 = s.rand(L, 99)
    fx, ft = s.fn(), s.fn()
    fx.upload(L, x0)
    r = H.estimate_radius(s.A, fx, ft, L, 30)
    ro = O.power_iteration_radius(s.op, L, x0, 30)
    assert abs(r - ro) < 1e-10 * ro


@pytest.mark.parametrize("dtype,tol", [("float32", 1e-5), ("float16", 5e-3)])
def test_low_precision_storage_apply(ctx, dtype, tol):
    L = 4
    s = Setup(ctx, "cube_6", L, L, dtype=dtype)
    x = s.rand(L, 4)
    fx, fy = s.fn(), s.fn()
    fx.upload(L, x)
    s.A.apply(fx, fy, L, O.INNER)
    xq = fx.download(L)  # quantised input as stored
    ref = s.op.apply(xq, np.zeros_like(xq), L, O.INNER)
    mask = s.op.levels[L].owned_mask(O.INNER)
    assert relerr(fy.download(L), ref, mask) < tol
    f64 = H.P1Function("d", s.pm, L, L, ctx, "float64")
    f64.copyFrom(fy, L)
    assert relerr(f64.download(L), fy.download(L), mask) == 0.0


def test_errors_are_reported(ctx):
    s = Setup(ctx, "cube_6", 2, 3)
    f = s.fn()
    with pytest.raises(H.HybError):
        s.A.apply(f, f, 2, O.ALL)  # src == dst
    g = s.fn()
    with pytest.raises(H.HybError):
        s.A.apply(f, g, 5, O.ALL)  # level out of range
    h = H.P1Function("h", s.pm, 2, 3, ctx, "float32")
    with pytest.raises(H.HybError):
        s.A.apply(f, h, 2, O.ALL)  # mixed value types


def test_graph_replay_after_context_scratch_grows():
    """A captured V-cycle graph keeps the addresses of the context's reduction partials (the coarse
    CG's dot products are inside the graph).  When a later, larger reduction on the same context
    needs a bigger partials buffer, the old buffer must stay valid for the graph: cycles replayed
    after the growth give the same bits as on a context where nothing grew."""
    L = 4
    runs = []
    for grow in (False, True):
        c = H.Context(0)
        s = Setup(c, "cube_6", 0, L)
        b = s.rand(L, 21, O.INNER)
        fx, fb = s.fn(), s.fn()
        fb.upload(L, b)
        gmg = H.GeometricMultigridSolver(c, s.A, 0, L, preSmoothSteps=2, postSmoothSteps=2, use_graph=True)
        h1 = gmg.solve_cycles(fx, fb, L, 3)  # the graph is captured during these cycles
        if grow:
            before = c.scratch_bytes
            # about 105,000 block partials, more than the 65,536 reserved at the start
            big = H.PrimitiveStorage.spherical_shell(5, 3, 0.55, 1.0, ctx=c)
            f = H.P1Function("f", big, 5, 5, c)
            f.fill_random(5, 3)
            f.dotGlobal(f, 5, H.All)
            assert c.scratch_bytes > before
        h2 = gmg.solve_cycles(fx, fb, L, 3)  # replays the captured graph
        runs.append((h1, h2, fx.download(L)))
        c.close()
    np.testing.assert_array_equal(runs[0][1], runs[1][1])
    np.testing.assert_array_equal(runs[0][2], runs[1][2])
