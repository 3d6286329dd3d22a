"""GPU parity of the P2-P1 Taylor-Hood Stokes path (P2P1ElementwiseBlendingStokesOperator blocks with
the velocity block -div(eta grad) per component, the inverted PSPG diagonal, the Uzawa smoother and
the Uzawa multigrid) against the oracle assembled from the same element integrals (pinned to the
reference's p2_to_p1_div_*_blending_q2, p1_to_p2_divt_*_blending_q2 and p1_tet_pspg_tet forms on the
CPU).

Tolerances: blocks, apply and one Uzawa step within 1e-12 relative (max norm over the velocity's inner
DoFs and all pressure DoFs); V-cycle residual-reduction factors within 1e-6."""

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O
from tests import meshes as M

pytestmark = pytest.mark.gpu

ETA = ("radial", 2.99, 1.0, 0.45)


def _eta(case):
    """The radial viscosity of the shell configuration; on the unit cube (radii up to sqrt 3, where that
    profile spans five orders of magnitude and the unscaled Uzawa pressure step diverges) eta = 1."""
    return (ETA, O.k_radial(2.99, 1.0, 0.45)) if case == "shell" else (None, lambda P: np.ones(len(P)))


def _setup(ctx, case, minL, maxL, block="laplace"):
    coords, tets = M.cube_6() if case == "cube" else O.mesh_spherical_shell(3, 2, 0.55, 1.0)
    om = O.MacroMesh(coords, tets)
    bl = "shell" if case == "shell" else None
    S = O.P2P1Stokes(om, minL, maxL, _eta(case)[1], blending=bl, full_viscous=block == "full_viscous")
    S.block = block
    S.case = case
    pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
    return S, pm, bl


def _vel(S, L, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(3):
        x = np.zeros(S.ulev[L].size)
        m = S.umask(L)
        x[m] = rng.uniform(-1, 1, m.sum())
        out.append(S.ulev[L].sync(x))
    return out


def _pres(S, L, seed):
    rng = np.random.default_rng(seed)
    x = np.zeros(S.plev[L].size)
    m = S.pmask(L)
    x[m] = rng.uniform(-1, 1, m.sum())
    return S.plev[L].sync(x)


def _fns(pm, ctx, minL, maxL):
    u = [H.P2Function("u%d" % k, pm, minL, maxL, ctx) for k in range(3)]
    p = H.P1Function("p", pm, minL, maxL, ctx)
    return u, p


def _relerr(a, b, mask):
    return np.abs(a[mask] - b[mask]).max() / max(np.abs(b[mask]).max(), 1e-300)


@pytest.mark.parametrize("case,L", [("cube", 1), ("cube", 2), ("shell", 1)])
def test_stokes_blocks_match_oracle(ctx, case, L):
    S, pm, bl = _setup(ctx, case, L, L)
    u0, p0 = _vel(S, L, 1), _pres(S, L, 2)
    u, p = _fns(pm, ctx, L, L)
    for k in range(3):
        u[k].upload(L, u0[k])
    p.upload(L, p0)
    D = H.P2ToP1ElementwiseBlendingDivOperator(pm, L, L, ctx, blending=bl)
    dp = H.P1Function("dp", pm, L, L, ctx)
    D.apply(u, dp, L, H.All)
    assert _relerr(dp.download(L), S.div(u0, L), S.pmask(L)) < 1e-12
    du = [H.P2Function("du%d" % k, pm, L, L, ctx) for k in range(3)]
    D.applyTranspose(p, du, L, H.Inner)
    ref = S.divt(p0, L)
    for k in range(3):
        assert _relerr(du[k].download(L), ref[k], S.umask(L)) < 1e-12
    # divT adds onto a vector and is the transpose of div: <div u, p> = <u, divT p>
    lhs = float(np.dot(dp.download(L)[S.pmask(L)], p0[S.pmask(L)]))
    rhs = sum(float(np.dot(u0[k][S.umask(L)], du[k].download(L)[S.umask(L)])) for k in range(3))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)
    P = H.P1PSPGOperator(pm, L, L, ctx)
    inv = H.P1Function("inv", pm, L, L, ctx)
    P.getInverseDiagonalValues(inv, L, H.All)
    assert _relerr(inv.download(L), S.sinv[L], S.pmask(L)) < 1e-12


def _solver(ctx, pm, S, bl, minL, maxL, **kw):
    if S.Vop is None:
        radii = [O.power_iteration_radius(S.Aop, l, np.random.default_rng(40 + l).uniform(-1, 1, S.ulev[l].size), 20)
                 for l in range(minL, maxL + 1)]
    else:
        radii = [O.power_iteration_radius_vec(S.Vop, l, [np.random.default_rng(40 + l + 7 * k).uniform(-1, 1, S.ulev[l].size)
                                                         for k in range(3)], 20)
                 for l in range(minL, maxL + 1)]
    st = H.StokesUzawaMultigrid(ctx, pm, minL, maxL, viscosity=_eta(S.case)[0], blending=bl,
                                velocity_block=S.block, **kw)
    st.set_velocity_radii(radii)
    return st, {l: radii[l - minL] for l in range(minL, maxL + 1)}


@pytest.mark.parametrize("block", ["laplace", "full_viscous"])
@pytest.mark.parametrize("case", ["cube", "shell"])
def test_stokes_apply_and_uzawa_step(ctx, case, block):
    L = 2 if case == "cube" else 1
    S, pm, bl = _setup(ctx, case, 0, L, block)
    st, radii = _solver(ctx, pm, S, bl, 0, L)
    u0, p0 = _vel(S, L, 3), _pres(S, L, 4)
    bu0, bp0 = _vel(S, L, 5), _pres(S, L, 6)
    u, p = _fns(pm, ctx, 0, L)
    bu, bp = _fns(pm, ctx, 0, L)
    du, dp = _fns(pm, ctx, 0, L)
    for k in range(3):
        u[k].upload(L, u0[k])
        bu[k].upload(L, bu0[k])
    p.upload(L, p0)
    bp.upload(L, bp0)
    st.apply(u, p, du, dp, L)
    rdu, rdp = S.apply(u0, p0, L)
    for k in range(3):
        assert _relerr(du[k].download(L), rdu[k], S.umask(L)) < 1e-12
    assert _relerr(dp.download(L), rdp, S.pmask(L)) < 1e-12
    r = st.residual_norm(u, p, bu, bp, L)
    rr = S.residual_norm(u0, p0, bu0, bp0, L)
    assert abs(r - rr) <= 1e-12 * rr
    st.uzawa_smooth(u, p, bu, bp, L)
    ru, rp = S.uzawa(u0, p0, bu0, bp0, L, radii[L])
    for k in range(3):
        assert _relerr(u[k].download(L), ru[k], S.umask(L)) < 1e-12
    assert _relerr(p.download(L), rp, S.pmask(L)) < 1e-12


@pytest.mark.parametrize("block", ["laplace", "full_viscous"])
@pytest.mark.parametrize("case", ["cube", "shell"])
def test_stokes_vcycle_factors(ctx, case, block):
    L = 3 if case == "cube" else 2
    S, pm, bl = _setup(ctx, case, 0, L, block)
    st, radii = _solver(ctx, pm, S, bl, 0, L)
    bu0, bp0 = _vel(S, L, 7), np.zeros(S.plev[L].size)
    u, p = _fns(pm, ctx, 0, L)
    bu, bp = _fns(pm, ctx, 0, L)
    for k in range(3):
        bu[k].upload(L, bu0[k])
    bp.upload(L, bp0)
    hist = st.solve(u, p, bu, bp, L, 3)
    uo, po = [np.zeros(S.ulev[L].size) for _ in range(3)], np.zeros(S.plev[L].size)
    ref = [S.residual_norm(uo, po, bu0, bp0, L)]
    for _ in range(3):
        uo, po = S.vcycle(uo, po, bu0, bp0, L, radii)
        ref.append(S.residual_norm(uo, po, bu0, bp0, L))
    ref = np.array(ref)
    np.testing.assert_allclose(hist[0], ref[0], rtol=1e-12)
    np.testing.assert_allclose(hist[1:] / hist[:-1], ref[1:] / ref[:-1], rtol=0, atol=1e-6)
    assert hist[-1] < hist[0]


@pytest.mark.parametrize("block", ["laplace", "full_viscous"])
@pytest.mark.parametrize("inner", ["float32"])
def test_stokes_mixed_precision_reaches_fp64_accuracy(ctx, inner, block):
    """FP64 defect correction around FP32 / FP16 Uzawa V-cycles reaches the same relative residual
    (1e-6; the Uzawa multigrid's asymptotic factor on this shell is about 0.84) and the FP64 V-cycle
    solution to within the residual level (1e-4 relative, max norm, velocity)."""
    L = 2
    S, pm, bl = _setup(ctx, "shell", 0, L)
    bu0 = _vel(S, L, 9)
    u, p = _fns(pm, ctx, 0, L)
    bu, bp = _fns(pm, ctx, 0, L)
    for k in range(3):
        bu[k].upload(L, bu0[k])
    st = H.StokesUzawaMultigrid(ctx, pm, 0, L, viscosity=ETA, blending=bl, velocity_block=block)
    hist = st.solve(u, p, bu, bp, L, 120, rtol=1e-6)
    assert hist[-1] < 1e-6 * hist[0]
    ui = [H.P2Function("ui%d" % k, pm, 0, L, ctx) for k in range(3)]
    pi = H.P1Function("pi", pm, 0, L, ctx)
    inner_solver = H.StokesUzawaMultigrid(ctx, pm, 0, L, viscosity=ETA, blending=bl, velocity_block=block)
    mh = st.mixed_solve(inner_solver, ui, pi, bu, bp, L, max_outer=120, rtol=1e-6, inner_dtype=inner)
    assert mh[-1] < 1e-6 * mh[0]
    m = S.umask(L)
    for k in range(3):
        a, b = ui[k].download(L)[m], u[k].download(L)[m]
        assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max()


def test_stokes_mixed_refuses_fp16(ctx):
    """FP16 inner cycles are refused (the inverted PSPG diagonal leaves the FP16 range)."""
    L = 1
    S, pm, bl = _setup(ctx, "cube", 0, L)
    u, p = _fns(pm, ctx, 0, L)
    bu, bp = _fns(pm, ctx, 0, L)
    st = H.StokesUzawaMultigrid(ctx, pm, 0, L)
    inner = H.StokesUzawaMultigrid(ctx, pm, 0, L)
    with pytest.raises(H.HybError):
        st.mixed_solve(inner, u, p, bu, bp, L, inner_dtype="float16")


def test_stokes_full_viscous_own_radii_converge(ctx):
    """Without given radii the solver estimates them by the power iteration on the coupled block."""
    L = 2
    S, pm, bl = _setup(ctx, "cube", 0, L, "full_viscous")
    st = H.StokesUzawaMultigrid(ctx, pm, 0, L, viscosity=_eta("cube")[0], blending=bl, velocity_block="full_viscous")
    bu0 = _vel(S, L, 9)
    u, p = _fns(pm, ctx, 0, L)
    bu, bp = _fns(pm, ctx, 0, L)
    for k in range(3):
        bu[k].upload(L, bu0[k])
    hist = st.solve(u, p, bu, bp, L, 6)
    assert np.all(hist[1:] / hist[:-1] < 0.9)
    assert hist[-1] < 1e-2 * hist[0]


def test_stokes_lumped_mass_scaling_uzawa_step_and_relaxation_estimate(ctx):
    """The pressure update scaled by the inverse lumped pressure mass weighted by 1/eta (blended shell,
    radial viscosity): one Uzawa step matches the oracle within 1e-12 with the same omega; the
    relaxation estimate (power iteration on |S|^-1 B A~^-1 B^T, estimateUzawaRelaxationParameter) gives a
    positive radius, and the Uzawa multigrid with omega = 1/radius reduces the residual by at least a
    factor 2 in every one of four V-cycles."""
    L = 1
    coords, tets = O.mesh_spherical_shell(3, 2, 0.55, 1.0)
    om = O.MacroMesh(coords, tets)
    S = O.P2P1Stokes(om, 0, L, _eta("shell")[1], blending="shell", pressure_scaling="lumped_mass")
    S.block, S.case = "laplace", "shell"
    pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
    st, radii = _solver(ctx, pm, S, "shell", 0, L, pressure_scaling="lumped_mass")
    omega = 1.7
    st.set_omega(omega)
    u0, p0 = _vel(S, L, 3), _pres(S, L, 4)
    bu0, bp0 = _vel(S, L, 5), _pres(S, L, 6)
    u, p = _fns(pm, ctx, 0, L)
    bu, bp = _fns(pm, ctx, 0, L)
    for k in range(3):
        u[k].upload(L, u0[k])
        bu[k].upload(L, bu0[k])
    p.upload(L, p0)
    bp.upload(L, bp0)
    st.uzawa_smooth(u, p, bu, bp, L)
    ru, rp = S.uzawa(u0, p0, bu0, bp0, L, radii[L], omega=omega)
    for k in range(3):
        assert _relerr(u[k].download(L), ru[k], S.umask(L)) < 1e-12
    assert _relerr(p.download(L), rp, S.pmask(L)) < 1e-12
    # estimate and multigrid on two levels more
    L2 = 2
    S2 = O.P2P1Stokes(om, 0, L2, _eta("shell")[1], blending="shell", pressure_scaling="lumped_mass")
    S2.block, S2.case = "laplace", "shell"
    st2, _ = _solver(ctx, pm, S2, "shell", 0, L2, pressure_scaling="lumped_mass")
    rho = st2.estimate_relaxation(1, 20, 2)
    assert 0.0 < rho < 10.0
    st2.set_omega(1.0 / rho)
    u, p = _fns(pm, ctx, 0, L2)
    bu, bp = _fns(pm, ctx, 0, L2)
    bu0 = _vel(S2, L2, 7)
    for k in range(3):
        bu[k].upload(L2, bu0[k])
    hist = st2.solve(u, p, bu, bp, L2, 4)
    assert (hist[1:] / hist[:-1]).max() < 0.5, hist
