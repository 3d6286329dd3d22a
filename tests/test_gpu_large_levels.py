"""GPU parity of the cell-interior sweep at levels 7 and 8, the sizes the benchmark runs.

The oracle's assembled operator does not fit at these levels, so the reference values come from
oracle.LargeLevelConstantOperator: cell interiors through the reference's own compiled
apply_3D_macrocell_vertexdof_to_vertexdof_replace kernel (oracle/_ref), face, edge and vertex owners
as the sum of the one-sided stencils of their neighbour cells.

Tolerances as in test_gpu_p1: FP64 within 1e-12 relative (max norm over owned DoFs), FP32 storage
within 1e-5 and FP16 storage within 5e-3 of the FP64 values on the stored inputs."""

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O
from oracle import ref as R
from tests import meshes as M

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")]

FLAG = O.INNER | O.NEUMANN | O.FREESLIP


def relerr(a, b, mask):
    return np.abs(a[mask] - b[mask]).max() / max(np.abs(b[mask]).max(), 1e-300)


class Big:
    """One mesh at one large level: the oracle operator and the GPU operator."""

    def __init__(self, ctx, name, L):
        coords, tets = M.ALL[name]()
        self.om = O.MacroMesh(coords, tets)
        self.op = O.LargeLevelConstantOperator(self.om, L, interior_kernel=R.cell_apply)
        self.lev = self.op.levels[L]
        self.pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
        self.A = H.P1ConstantLaplaceOperator(self.pm, L - 1, L, ctx)
        self.ctx, self.L = ctx, L
        self.copies = self.lev.copy_map()

    def fn(self, dtype="float64", name="f", min_level=None):
        return H.P1Function(name, self.pm, self.L if min_level is None else min_level, self.L, self.ctx, dtype)

    def rand(self, seed, flag=O.ALL):
        rng = np.random.default_rng(seed)
        x = np.zeros(self.lev.size)
        m = self.lev.owned_mask(flag)
        x[m] = rng.uniform(-1, 1, m.sum())
        return self.lev.sync(x)

    def assert_copies(self, vec):
        d, s = self.copies
        np.testing.assert_array_equal(vec[d], vec[s])


@pytest.fixture(scope="module")
def cube8(ctx):
    return Big(ctx, "cube_6", 8)


def test_apply_level8_matches_reference_kernel(ctx, cube8):
    """The benchmark's workload: FP64 apply on the six-tetrahedra cube at level 8, Replace and Add,
    flags Inner and All."""
    s, L = cube8, 8
    x, y0 = s.rand(81), s.rand(82)
    fx, fy = s.fn(name="x"), s.fn(name="y")
    fx.upload(L, x)
    mask = s.lev.owned_mask(O.ALL)
    for flag in (O.INNER, O.ALL):
        fy.upload(L, y0)
        s.A.apply(fx, fy, L, flag, H.Replace)
        ref = s.op.apply(x, y0.copy(), L, flag)
        got = fy.download(L)
        assert relerr(got, ref, mask) < 1e-12
        s.assert_copies(got)
        s.A.apply(fx, fy, L, flag, H.Add)
        ref2 = s.op.apply(x, ref.copy(), L, flag, add=True)
        assert relerr(fy.download(L), ref2, mask) < 1e-12


def test_residual_and_jacobi_level8(ctx, cube8):
    s, L = cube8, 8
    x, b = s.rand(83), s.rand(84)
    fx, fb, ft = s.fn(name="x"), s.fn(name="b"), s.fn(name="t")
    fx.upload(L, x)
    fb.upload(L, b)
    got = H.residual_norm(s.A, fx, fb, ft, L)
    r = b - s.op.full_apply(x)
    m = s.lev.owned_mask(FLAG)
    ref = float(np.sqrt(np.dot(r[m], r[m])))
    assert abs(got - ref) <= 1e-12 * ref
    fd = s.fn(name="d")
    s.A.smooth_jac(fd, fb, fx, 0.6, L, FLAG)
    ref = s.op.smooth_jac(np.zeros_like(x), b, x, 0.6, L, FLAG)
    got = fd.download(L)
    assert relerr(got, ref, s.lev.owned_mask(FLAG)) < 1e-12
    s.assert_copies(got)


@pytest.mark.parametrize("dtype,tol", [("float32", 1e-5), ("float16", 5e-3)])
def test_low_precision_apply_level8(ctx, cube8, dtype, tol):
    s, L = cube8, 8
    fx, fy = s.fn(dtype, "x"), s.fn(dtype, "y")
    fx.upload(L, s.rand(85))
    s.A.apply(fx, fy, L, O.INNER)
    xq = fx.download(L)  # the stored (rounded) input
    ref = s.op.apply(xq, np.zeros_like(xq), L, O.INNER)
    assert relerr(fy.download(L), ref, s.lev.owned_mask(O.INNER)) < tol


@pytest.mark.parametrize("name", ["octahedron_8", "cube_2x1x1"])
def test_apply_and_chebyshev_level7(ctx, name):
    """Other cell shapes and counts at level 7; the Chebyshev smoother's three fused epilogues (first,
    middle, last step) through GeometricMultigridSolver.smooth with a fixed spectral radius."""
    L = 7
    s = Big(ctx, name, L)
    x, b = s.rand(71), s.rand(72)
    fx, fy, fb = s.fn(name="x", min_level=L - 1), s.fn(name="y"), s.fn(name="b", min_level=L - 1)
    fx.upload(L, x)
    s.A.apply(fx, fy, L, O.ALL)
    mask = s.lev.owned_mask(O.ALL)
    assert relerr(fy.download(L), s.op.apply(x, np.zeros_like(x), L, O.ALL), mask) < 1e-12
    fb.upload(L, b)
    radius = 2.3
    gmg = H.GeometricMultigridSolver(ctx, s.A, L - 1, L, smoother="chebyshev", chebyshev_order=3, use_graph=False)
    gmg.set_radii([radius, radius])
    gmg.smooth(fx, fb, L, 2)
    g = O.GMG(s.op, None, L, L, smoother="chebyshev", cheb_order=3, cheb_radii={L: radius})
    ref = x.copy()
    for _ in range(2):
        g.chebyshev_step(ref, b, L)
    got = fx.download(L)
    assert relerr(got, ref, mask) < 1e-12
    s.assert_copies(got)
