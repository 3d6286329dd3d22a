"""GPU parity of the full viscous velocity block (P2ElementwiseBlendingFullViscousOperator: the nine
forms p2_full_stokesvar_{i}_{j}_blending_q3, applied matrix-free) against the oracle assembled from
the same element integrals (pinned to the reference forms on the CPU).

Tolerances: FP64 apply and inverse diagonal within 1e-12 relative (max norm over owned DoFs, per
component); FP32 storage within 2e-6 of the FP64 oracle applied to the rounded input."""

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O
from tests import meshes as M
from tests.test_gpu_p2 import _rand, _relerr, lev_pack, lev_unpack

pytestmark = pytest.mark.gpu

MU_SPEC = ("expsin", 0.5, (0.13, 0.27, 0.41))


def _setup(ctx, case, L, mu=MU_SPEC):
    coords, tets = M.cube_6() if case == "cube" else O.mesh_spherical_shell(3, 2, 0.55, 1.0)
    om = O.MacroMesh(coords, tets)
    bl = "shell" if case == "shell" else None
    mufun = O.k_expsin(mu[1], mu[2]) if mu[0] == "expsin" else O.k_radial(*mu[1:])
    op = O.P2FullViscous(om, L, L, mufun, blending=bl)
    pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
    A = H.P2ElementwiseBlendingFullViscousOperator(pm, L, L, ctx, viscosity=mu, blending=bl)
    return op, pm, A


@pytest.mark.parametrize("case", ["cube", "shell"])
@pytest.mark.parametrize("L", [1, 2, 3])
def test_full_viscous_apply_and_diagonal_match_oracle(ctx, case, L):
    op, pm, A = _setup(ctx, case, L)
    lev = op.levels[L]
    u = [_rand(lev, 10 + k) for k in range(3)]
    y0 = [_rand(lev, 20 + k) for k in range(3)]
    fu = [H.P2Function("u%d" % k, pm, L, L, ctx) for k in range(3)]
    fy = [H.P2Function("y%d" % k, pm, L, L, ctx) for k in range(3)]
    for k in range(3):
        fu[k].upload(L, lev_pack(pm, lev, L, u[k]))
    mask = lev.owned_mask(O.ALL)
    d, s = lev.copy_map()
    for flag in (O.INNER, O.ALL):
        for k in range(3):
            fy[k].upload(L, lev_pack(pm, lev, L, y0[k]))
        A.apply(fu, fy, L, flag, H.Replace)
        ref = op.apply(u, [v.copy() for v in y0], L, flag)
        got = [lev_unpack(pm, lev, L, fy[k].download(L)) for k in range(3)]
        for k in range(3):
            assert _relerr(got[k], ref[k], mask) < 1e-12, (flag, k)
            np.testing.assert_array_equal(got[k][d], got[k][s])
        A.apply(fu, fy, L, flag, H.Add)
        ref2 = op.apply(u, [v.copy() for v in ref], L, flag, add=True)
        for k in range(3):
            assert _relerr(lev_unpack(pm, lev, L, fy[k].download(L)), ref2[k], mask) < 1e-12
    fd = [H.P2Function("d%d" % k, pm, L, L, ctx) for k in range(3)]
    A.getInverseDiagonalValues(fd, L)
    for k in range(3):
        assert _relerr(lev_unpack(pm, lev, L, fd[k].download(L)), op.invdiag[L][k], mask) < 1e-12


def test_full_viscous_radial_viscosity_fp32(ctx):
    """The radial viscosity of the mantle configuration, FP32 storage and accumulation."""
    L = 2
    mu = ("radial", 2.99, 1.0, 0.45)
    op, pm, A = _setup(ctx, "shell", L, mu)
    lev = op.levels[L]
    u = [_rand(lev, 30 + k) for k in range(3)]
    fu = [H.P2Function("u%d" % k, pm, L, L, ctx, dtype="float32") for k in range(3)]
    fy = [H.P2Function("y%d" % k, pm, L, L, ctx, dtype="float32") for k in range(3)]
    for k in range(3):
        fu[k].upload(L, lev_pack(pm, lev, L, u[k]))
    uq = [lev_unpack(pm, lev, L, fu[k].download(L)) for k in range(3)]
    A.apply(fu, fy, L, O.INNER)
    ref = op.apply(uq, [np.zeros(lev.size) for _ in range(3)], L, O.INNER)
    mask = lev.owned_mask(O.INNER)
    for k in range(3):
        assert _relerr(lev_unpack(pm, lev, L, fy[k].download(L)), ref[k], mask) < 2e-6


def test_full_viscous_refused_by_scalar_entry_points(ctx):
    op, pm, A = _setup(ctx, "cube", 1)
    f, g = H.P2Function("f", pm, 1, 1, ctx), H.P2Function("g", pm, 1, 1, ctx)
    with pytest.raises(H.HybError, match="block operators"):
        H._check(H.lib().hyb_op_apply(A.h, f.h, g.h, 1, O.INNER, H.Replace))
