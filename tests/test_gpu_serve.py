"""GPU tests of the solve server (continuous admission into resident multigrid slots).

Every slot owns its vectors, hierarchy, captured cycle graph and stream, and every reduction is
deterministic (no atomics), so a request must give the SAME bits whether it ran alone or inside a
mix of concurrent requests, and the same bits as the plain solver API driven with the same
parameters (Chebyshev(3) V(3,3) cycles, 20 power iterations, stop at ||r||/||r0|| < rtol)."""

import numpy as np
import pytest

import hyteg_b200 as H

pytestmark = pytest.mark.gpu

K_SPEC = ("expsin", 0.5, (0.13, 0.27, 0.41))


def _meshes(ctx):
    return {"cube": H.PrimitiveStorage.cuboid(ctx=ctx), "shell": H.PrimitiveStorage.spherical_shell(3, 2, 0.55, 1.0, ctx=ctx)}


def _requests():
    # (mesh, level, kind, k, blending, seed, mixed)
    return [
        ("cube", 4, "laplace", None, None, 11, False),
        ("cube", 5, "laplace", None, None, 12, False),
        ("shell", 3, "divkgrad", K_SPEC, "shell", 13, False),
        ("cube", 4, "laplace", None, None, 14, True),
        ("shell", 3, "divkgrad", 2.0, "shell", 15, False),
        ("cube", 5, "laplace", None, None, 16, True),
        ("cube", 4, "divkgrad", K_SPEC, None, 17, False),
        ("cube", 4, "laplace", None, None, 18, False),
    ]


def _submit(srv, meshes, req, rtol=1e-8):
    m, L, kind, k, bl, seed, mixed = req
    return srv.submit(meshes[m], L, kind=kind, k=k, blending=bl, seed=seed, rtol=rtol, max_cycles=40, mixed=mixed,
                      want_solution=True)


def _solve_alone(ctx, meshes, req):
    srv = H.SolveServer(ctx, max_slots=4)
    rid = _submit(srv, meshes, req)
    srv.drain()
    st = srv.status(rid)
    x = srv.solution(rid).copy()
    srv.close()
    return st, x


def test_serve_mix_equals_alone(ctx):
    meshes = _meshes(ctx)
    reqs = _requests()
    srv = H.SolveServer(ctx, max_slots=6)
    ids = [_submit(srv, meshes, r) for r in reqs]
    srv.drain()
    for r, rid in zip(reqs, ids):
        st = srv.status(rid)
        assert st["state"] == H.CONVERGED, (r, st)
        assert st["rel_res"] < 1e-8
        assert st["t_arrival"] <= st["t_admit"] <= st["t_done"]
        st1, x1 = _solve_alone(ctx, meshes, r)
        assert st1["cycles"] == st["cycles"], r
        np.testing.assert_array_equal(srv.solution(rid), x1)
    srv.close()


def test_serve_matches_plain_solver(ctx):
    """A plain FP64 request reproduces GeometricMultigridSolver.solve_cycles bit for bit."""
    pm = H.PrimitiveStorage.cuboid(ctx=ctx)
    L = 5
    srv = H.SolveServer(ctx, max_slots=2)
    rid = srv.submit(pm, L, seed=7, rtol=1e-8, max_cycles=40, want_solution=True)
    srv.drain()
    st = srv.status(rid)
    A = H.P1ConstantLaplaceOperator(pm, 0, L, ctx)
    gmg = H.GeometricMultigridSolver(ctx, A, 0, L, 3, 3, smoother="chebyshev", chebyshev_order=3, power_iterations=20)
    x = H.P1Function("x", pm, 0, L, ctx)
    b = H.P1Function("b", pm, 0, L, ctx)
    b.fill_random(L, 7)
    hist = gmg.solve_cycles(x, b, L, 40, rtol=1e-8)
    assert len(hist) - 1 == st["cycles"]
    assert abs(hist[-1] / hist[0] - st["rel_res"]) <= 1e-12 * max(1e-30, st["rel_res"])
    np.testing.assert_array_equal(x.download(L), srv.solution(rid))
    srv.close()


def test_serve_mixed_precision_reaches_fp64_accuracy(ctx):
    pm = H.PrimitiveStorage.cuboid(ctx=ctx)
    L = 5
    srv = H.SolveServer(ctx, max_slots=2)
    a = srv.submit(pm, L, seed=3, rtol=1e-9, max_cycles=40, want_solution=True)
    b = srv.submit(pm, L, seed=3, rtol=1e-9, max_cycles=40, mixed=True, want_solution=True)
    srv.drain()
    assert srv.status(a)["state"] == H.CONVERGED and srv.status(b)["state"] == H.CONVERGED
    xa, xb = srv.solution(a), srv.solution(b)
    assert np.abs(xa - xb).max() <= 1e-7 * np.abs(xa).max()
    srv.close()


def _slot_bytes(pm, L, divkgrad):
    """The server's footprint estimate of a plain slot: ten FP64 vectors over all levels, plus the
    stored matrices of a div-k-grad operator (assembled stencils: 15 values per DoF)."""
    vec = sum(pm.packed_size(l) for l in range(L + 1)) * 8 * 10
    mats = sum(pm.packed_size(l) * 15 for l in range(L + 1)) * 8
    return vec + (mats if divkgrad else 0)


def test_serve_budget_evicts_and_rejects(ctx):
    pm = H.PrimitiveStorage.cuboid(ctx=ctx)
    # room for the div-k-grad slot but not for it and a Laplace slot together: every switch of
    # operator evicts the idle slot of the other kind
    budget = _slot_bytes(pm, 4, True) + 0.5 * _slot_bytes(pm, 4, False)
    srv = H.SolveServer(ctx, max_slots=8, hbm_budget_bytes=budget)
    ids = [srv.submit(pm, 4, kind="divkgrad" if i % 2 else "laplace", seed=i, rtol=1e-8, want_solution=True) for i in range(4)]
    srv.drain()
    for i, rid in enumerate(ids):
        assert srv.status(rid)["state"] == H.CONVERGED
    with pytest.raises(H.HybError):
        srv.submit(pm, 7, seed=1)  # can never fit the budget
    srv.close()


def _batched(ctx, meshes, reqs, width=4, rtol=1e-8):
    srv = H.SolveServer(ctx, max_slots=8, batch_width=width)
    ids = [_submit(srv, meshes, r, rtol=rtol) for r in reqs]
    srv.drain()
    out = [(srv.status(rid), srv.solution(rid).copy()) for rid in ids]
    srv.close()
    return out


def test_serve_batches_match_single_solves(ctx):
    """Batch slots (FP64 requests of one key share one multigrid on disjoint copies of the mesh): every
    request converges, and its solution agrees with the one-slot solve within the tolerance's reach
    (relative max-norm difference below 1e-6 at rtol 1e-8: the two runs use spectral-radius estimates
    from different start vectors, and on the shell the coarse CG couples the copies)."""
    meshes = _meshes(ctx)
    reqs = [r for r in _requests() if not r[6]] + [("cube", 4, "laplace", None, None, 19, False),
                                                   ("cube", 4, "laplace", None, None, 20, False)]
    got = _batched(ctx, meshes, reqs)
    for r, (st, x) in zip(reqs, got):
        assert st["state"] == H.CONVERGED, (r, st)
        assert st["rel_res"] < 1e-8
        st1, x1 = _solve_alone(ctx, meshes, r)
        assert np.abs(x - x1).max() <= 1e-6 * np.abs(x1).max(), r


def test_serve_batch_place_alone_equals_mix(ctx):
    """On the six-tetrahedra cube (no free DoF on the coarsest level, so nothing couples the copies) a
    request gives the same bits alone in its batch and among other requests of the batch; on the shell
    the copies share the coarse CG's step lengths and the results agree within 1e-6."""
    meshes = _meshes(ctx)
    mix = [("cube", 4, "laplace", None, None, s, False) for s in (31, 32, 33, 34, 35)]
    together = _batched(ctx, meshes, mix, width=4)
    for r, (st, x) in zip(mix, together):
        st1, x1 = _batched(ctx, meshes, [r], width=4)[0]
        assert st1["cycles"] == st["cycles"], r
        np.testing.assert_array_equal(x, x1)
    shell = [("shell", 3, "divkgrad", K_SPEC, "shell", s, False) for s in (41, 42, 43)]
    together = _batched(ctx, meshes, shell, width=2)
    for r, (st, x) in zip(shell, together):
        st1, x1 = _batched(ctx, meshes, [r], width=2)[0]
        assert st["state"] == H.CONVERGED and st1["state"] == H.CONVERGED
        assert np.abs(x - x1).max() <= 1e-6 * np.abs(x1).max(), r


def test_serve_p2_requests(ctx):
    """P2 requests (elementwise div-k-grad on the blended shell, the P2 constant Laplacian on the cube)
    converge alone, and in a server with batch slots (where P2 requests keep one-solve slots) they give
    the same bits as alone."""
    meshes = _meshes(ctx)
    reqs = [("shell", 2, "p2_divkgrad", K_SPEC, "shell", 51, False), ("cube", 3, "p2_laplace", None, None, 52, False),
            ("cube", 3, "p2_laplace", None, None, 53, False), ("shell", 2, "p2_divkgrad", K_SPEC, "shell", 54, False)]
    single = []
    for r in reqs:
        st, x = _solve_alone(ctx, meshes, r)
        assert st["state"] == H.CONVERGED and st["rel_res"] < 1e-8, (r, st)
        single.append(x)
    got = _batched(ctx, meshes, reqs, width=2)
    for r, x1, (st, x) in zip(reqs, single, got):
        assert st["state"] == H.CONVERGED, (r, st)
        assert np.array_equal(x, x1), r
