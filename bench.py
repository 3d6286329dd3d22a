"""Benchmark of the P1 matrix-free multigrid path on B200.

Workload (one "step"): one application of the P1 constant-stencil Laplacian (flag Inner) on the
unit cube split into six macro-tetrahedra, refinement level 8 (16,974,593 DoFs, 16,581,375
inner), FP64 storage — the operator apply of the level-8 cube configuration.  The metric is MDoF/s
(inner DoFs x applies / s, ApplyBenchmark.cpp:104 of the reference).  Extra fields report one
FP64 V(3,3) Chebyshev(3) cycle on the same mesh and level.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: the path shards by macro-primitive but the multi-GPU exchange is not built yet, so N>1
runs N independent replicas (weak scaling), timed with CUDA events, max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

LEVEL = 8
METRIC = "MDoF/s apply (P1 constant-stencil Laplace, FP64)"
UNIT = "MDoF/s"
WORKLOAD = "P1 constant-stencil Laplace apply, unit cube 6 macro-tets, level 8, FP64, flag Inner"


def inner_dofs(L):
    n = 1 << L
    return (n - 1) ** 3


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--level", type=int, default=LEVEL)
    p.add_argument("--no-vcycle", action="store_true")
    p.add_argument("--no-mixed", action="store_true")
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--no-p2", action="store_true")
    p.add_argument("--no-stokes", action="store_true")
    p.add_argument("--no-config1", action="store_true")
    p.add_argument("--no-p2c", action="store_true")
    p.add_argument("--config4", action="store_true",
                   help="run configuration 4 as stated (P2-P1 Stokes on the shell (5,3) at level 5, FP32 inner / FP64 "
                        "outer Uzawa multigrid to rtol 1e-8; a few minutes) and print its own JSON line")
    p.add_argument("--config5", action="store_true",
                   help="run configuration 5 as stated (2000 requests, P1 or P2, cube or shell ntan 3/5 nrad 3, "
                        "levels 3-7) through the serving loop and print its own JSON line")
    p.add_argument("--config5-requests", type=int, default=2000,
                   help="length of the configuration-5 request stream (its first N requests; 2000 as stated)")
    p.add_argument("--config2", action="store_true",
                   help="run configuration 2 as stated (P2 div-k-grad on the shell (5,3) at level 6, Chebyshev(3) "
                        "V(3,3) to rtol 1e-10; about two minutes) and print its own JSON line")
    p.add_argument("--serve-requests", type=int, default=200)
    p.add_argument("--profile-vcycle", action="store_true",
                   help="run one FP64 and one FP32 V(3,3) Chebyshev(3) cycle of the level-8 cube without graph capture "
                        "between profiler start/stop (for ncu --profile-from-start off) and print their times")
    return p.parse_args()


def dist_setup(n):
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def job_rate(ms_local, units, world, device):
    """Whole-job throughput of one step timed on every rank: the slowest rank's time (max over ranks)
    and units x ranks / that time, in millions of units per second."""
    import torch

    t = torch.tensor([float(ms_local)], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(t.item())
    return ms_max, world * units / (ms_max * 1e-3) / 1e6


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=2)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the cell apply kernel from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "p1_cell_apply_cube_L8.json")
    try:
        with open(p) as f:
            return json.load(f).get("traffic_bytes_per_launch")
    except Exception:
        return None


def cpu_reference_apply(L, seconds=10.0, max_steps=None, threads=None):
    """The reference's own generated cell-apply kernel (oracle/_ref) on the six macro-cells, one
    macro-cell per OpenMP thread.  Returns (MDoF/s, applies, threads, seconds)."""
    import ctypes as C

    from oracle import hyteg_oracle as O
    from oracle import ref as R

    if not R.available():
        return None
    n = 1 << L
    size = O.tet_size(n + 1)
    rng = np.random.default_rng(0)
    ncell = 6
    src = [rng.uniform(-1, 1, size) for _ in range(ncell)]
    dst = [np.zeros(size) for _ in range(ncell)]
    st = np.tile(np.array([5.0] + [-0.5] * 8 + [0.25] * 6), ncell)
    dp = C.POINTER(C.c_double)
    sp = (dp * ncell)(*[a.ctypes.data_as(dp) for a in src])
    dpp = (dp * ncell)(*[a.ctypes.data_as(dp) for a in dst])
    threads = threads or min(ncell, os.cpu_count() or 1)
    lib = R.lib()
    lib.ref_cell_apply_many(ncell, dpp, sp, L, st.ctypes.data_as(dp), threads)  # warm-up
    t0 = time.perf_counter()
    k = 0
    while True:
        lib.ref_cell_apply_many(ncell, dpp, sp, L, st.ctypes.data_as(dp), threads)
        k += 1
        el = time.perf_counter() - t0
        if (max_steps and k >= max_steps) or (not max_steps and el >= seconds):
            break
    cell_inner = ncell * O.tet_size(n - 3) if n >= 4 else 0
    return cell_inner * k / el / 1e6, k, threads, el


def reference_parity(H, pm, x, y, L):
    """Checker for the timed apply: the largest difference between this level's cell interiors of
    y = A x and the reference's own compiled cell kernel (apply_3D_macrocell_vertexdof_to_vertexdof_
    replace, oracle/_ref) run on the same device input x, relative to the largest reference value.
    The stencil of each macro-cell comes from the oracle's element matrices."""
    from oracle import hyteg_oracle as O
    from oracle import ref as R

    if not R.available():
        return None
    nV, nE, nF, nC = pm.counts()
    coords = pm.vertex_coords()
    tets = np.array([pm.primitive_vertices(3, c) for c in range(nC)], dtype=np.int64)
    om = O.MacroMesh(coords, tets)
    offs, _ = pm.primitive_offsets(L)
    xs, ys = x.download(L), y.download(L)
    n = 1 << L
    size = O.tet_size(n + 1)
    pts = O.tet_points(n + 1)
    inner = (pts.min(axis=1) >= 1) & (pts.sum(axis=1) <= n - 1)
    worst = 0.0
    for c in range(nC):
        o = int(offs[nV + nE + nF + c])
        ref = R.cell_apply(np.ascontiguousarray(xs[o:o + size]), L, O.cell_stencils_by_mask(om, c, L)[0])
        d = np.abs(ys[o:o + size][inner] - ref[inner]).max() / max(np.abs(ref[inner]).max(), 1e-300)
        worst = max(worst, float(d))
    return worst


def config1_leg(H, ctx, L=5, cycles=10):
    """Configuration 1 as stated: P1 Poisson on the six-tetrahedra cube, level 5, rhs = mass matrix x
    interpolated 3 pi^2 sin(pi x) sin(pi y) sin(pi z), zero guess, V(2,2) weighted Jacobi 2/3, CG coarse
    solve to 1e-14 on level 0, ten cycles (graph-captured).  Reports the per-cycle residual reduction,
    the time per cycle and the FP64 apply rate on level 5 (a 0.3 MB vector: latency-bound, absolute
    times)."""
    import math

    import torch

    pm = H.PrimitiveStorage.cuboid(ctx=ctx)
    A = H.P1ConstantLaplaceOperator(pm, 0, L, ctx)
    M = H.P1ConstantMassOperator(pm, L, L, ctx)
    f, b, x = (H.P1Function(nm, pm, 0, L, ctx) for nm in ("f1", "b1", "x1"))
    pi = math.pi
    f.interpolate(lambda X, Y, Z: 3 * pi * pi * math.sin(pi * X) * math.sin(pi * Y) * math.sin(pi * Z), L, H.All)
    M.apply(f, b, L, H.All, H.Replace)
    gmg = H.GeometricMultigridSolver(ctx, A, 0, L, preSmoothSteps=2, postSmoothSteps=2, smoother="jacobi",
                                     relax=2.0 / 3.0, coarse_rtol=1e-14)
    gmg.solve_cycles(x, b, L, 2)  # set-up and graph capture
    best = None
    for _ in range(3):
        for lv in range(L + 1):
            x.interpolate(0.0, lv, H.All)
        ctx.synchronize()
        t0 = time.perf_counter()
        hist = gmg.solve_cycles(x, b, L, cycles)
        sec = time.perf_counter() - t0
        best = sec if best is None else min(best, sec)
    y = H.P1Function("y1", pm, L, L, ctx)
    for _ in range(10):
        A.apply(x, y, L, H.Inner)
    ctx.synchronize()
    n_ap = 200
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s = torch.cuda.ExternalStream(ctx.stream)
    e0.record(s)
    for _ in range(n_ap):
        A.apply(x, y, L, H.Inner)
    e1.record(s)
    e1.synchronize()
    ms_ap = e0.elapsed_time(e1) / n_ap
    return {"level": L, "inner_dofs": inner_dofs(L), "cycle": "V(2,2) weighted Jacobi 2/3, CG coarse level 0 to 1e-14",
            "rhs": "P1 mass x interpolated 3 pi^2 sin sin sin", "cycles": int(hist.size - 1),
            "factors": [float(v) for v in hist[1:] / hist[:-1]], "rel_residual": float(hist[-1] / hist[0]),
            "seconds_10_cycles": best, "ms_per_cycle": best * 1e3 / cycles,
            "apply_ms": ms_ap, "apply_mdofs": inner_dofs(L) / (ms_ap * 1e-3) / 1e6}


def mixed_precision_leg(H, ctx, pm, A, L, rtol=1e-10):
    """Configuration 3: time to ||r||/||r0|| < rtol (1e-10) from a zero guess: plain FP64 V(3,3) Chebyshev(3) cycles against
    FP64 defect correction around the same cycles in FP32 and FP16 storage (FP32 accumulation).
    Each solution's error is measured against an FP64 solution converged to 1e-13."""
    import torch

    b = H.P1Function("b_mp", pm, 0, L, ctx)
    b.fill_random(L, 2024)
    out = {"rtol": rtol, "level": L, "cycle": "V(3,3) Chebyshev(3), CG coarse level 0 (FP64)", "rhs": "seeded uniform [-1,1]"}
    gmg = H.GeometricMultigridSolver(ctx, A, 0, L, preSmoothSteps=3, postSmoothSteps=3, smoother="chebyshev",
                                     chebyshev_order=3, power_iterations=20)
    xr = H.P1Function("x_ref", pm, 0, L, ctx)
    gmg.solve_cycles(xr, b, L, 40, rtol=1e-13)
    x_ref = xr.download(L)
    nref = float(np.linalg.norm(x_ref))

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        ctx.synchronize()
        return r, time.perf_counter() - t0

    runs = {}
    x = H.P1Function("x_mp", pm, 0, L, ctx)
    # a solver instance serves one value type: one per inner precision
    solvers = {"fp64": gmg}
    for name in ("fp32", "fp16"):
        solvers[name] = H.GeometricMultigridSolver(ctx, A, 0, L, preSmoothSteps=3, postSmoothSteps=3, smoother="chebyshev",
                                                   chebyshev_order=3, power_iterations=20)
    for name in ("fp64", "fp32", "fp16"):
        best = None
        for rep in range(2):  # first run also captures the cycle graphs of this precision
            for lv in range(0, L + 1):
                x.interpolate(0.0, lv, H.All)
            if name == "fp64":
                hist, sec = timed(lambda: gmg.solve_cycles(x, b, L, 60, rtol=rtol))
            else:
                hist, sec = timed(lambda: solvers[name].mixed_solve(A, x, b, L, inner_dtype="float" + name[2:],
                                                                    inner_cycles=1, max_outer=60, rtol=rtol))
            if best is None or sec < best[1]:
                best = (hist, sec)
        hist, sec = best
        err = float(np.linalg.norm(x.download(L) - x_ref)) / nref
        runs[name] = {"seconds": sec, "cycles": len(hist) - 1, "rel_residual": float(hist[-1] / hist[0]),
                      "rel_error_vs_fp64_solution": err}
    for name in ("fp32", "fp16"):
        runs[name]["speedup_vs_fp64"] = runs["fp64"]["seconds"] / runs[name]["seconds"]
    out["runs"] = runs
    return out


def serving_leg(H, ctx, nreq=200, seed=7):
    """A bounded sample of the serving stream: `nreq` requests (Poisson arrivals at a rate above what
    the GPU sustains), each a P1 Poisson or div-k-grad solve on the 6-tet cube (levels 3-7) or the
    icosahedral shell ntan=3 (levels 3-5, shell blending for div-k-grad), k = exp(0.5 sin cos sin)
    with one of two phases, rtol 1e-8, mixed precision (FP32 inner, FP64 outer).  Every hierarchy is
    set up once before timing (warm slots).  Baselines: (1) sequential plain FP64 solves, the same
    requests one after another through the plain drop-in API, each building its operator (stored
    matrices for div-k-grad), solver and functions, solving and reading back its solution, as a user
    of the plain form solves a stream of different problems; (2) sequential warm FP64 solves on the
    server's resident hierarchies, one request at a time."""
    rng = np.random.default_rng(seed)
    meshes = {"cube": H.PrimitiveStorage.cuboid(ctx=ctx), "shell": H.PrimitiveStorage.spherical_shell(3, 2, 0.55, 1.0, ctx=ctx)}
    phases = [(0.13, 0.27, 0.41), (0.71, 0.05, 0.33)]
    reqs = []
    for i in range(nreq):
        m = "cube" if rng.random() < 0.5 else "shell"
        L = int(rng.integers(3, 8 if m == "cube" else 6))
        kind = "laplace" if rng.random() < 0.3 else "divkgrad"
        ph = phases[int(rng.integers(0, 2))]
        reqs.append((m, L, kind, ("expsin", 0.5, ph) if kind == "divkgrad" else None,
                     "shell" if (m == "shell" and kind == "divkgrad") else None, int(rng.integers(1, 2**31))))
    keys = sorted(set((r[0], r[1], r[2], r[3], r[4]) for r in reqs), key=str)

    def plain(reqs):
        t0 = time.perf_counter()
        ok, lat = 0, []
        for r in reqs:
            m, L, kind, kk, bl, seed = r
            ts = time.perf_counter()
            pm = meshes[m]
            if kind == "laplace":
                A = H.P1ConstantLaplaceOperator(pm, 0, L, ctx)
            else:
                A = H.P1ElementwiseBlendingDivKGradOperator(pm, 0, L, ctx, k=kk, blending=bl)
                A.computeAndStoreLocalElementMatrices()
            g = H.GeometricMultigridSolver(ctx, A, 0, L, 3, 3, smoother="chebyshev", chebyshev_order=3, power_iterations=20)
            x = H.P1Function("x", pm, 0, L, ctx)
            b = H.P1Function("b", pm, 0, L, ctx)
            b.fill_random(L, seed)
            hist = g.solve_cycles(x, b, L, 60, rtol=1e-8)
            x.download(L)
            ok += int(hist[-1] < 1e-8 * hist[0])
            g.close()
            del A, g, x, b
            lat.append(time.perf_counter() - ts)
        t1 = time.perf_counter()
        lat = np.cumsum(lat)  # every request arrives at t0 and waits for the ones before it
        return {"solves_per_s": len(reqs) / (t1 - t0), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "converged": ok, "seconds": t1 - t0}

    def run(mixed, sequential, width=1):
        srv = H.SolveServer(ctx, max_slots=4 * len(keys), batch_width=width)
        for k in keys:  # warm every slot (operator, radii, captured cycle graphs)
            srv.submit(meshes[k[0]], k[1], kind=k[2], k=k[3], blending=k[4], seed=1, rtol=1e-8, mixed=mixed)
        srv.drain()
        ctx.synchronize()
        ids = []
        t0 = srv.now()
        if sequential:
            for r in reqs:
                ids.append(srv.submit(meshes[r[0]], r[1], kind=r[2], k=r[3], blending=r[4], seed=r[5], rtol=1e-8,
                                      max_cycles=60, mixed=mixed))
                srv.drain()
        else:
            gaps = rng.exponential(0.0005, nreq)  # mean inter-arrival 0.5 ms
            arrivals = t0 + np.cumsum(gaps)
            i = 0
            while True:
                now = srv.now()
                while i < nreq and arrivals[i] <= now:
                    r = reqs[i]
                    ids.append(srv.submit(meshes[r[0]], r[1], kind=r[2], k=r[3], blending=r[4], seed=r[5], rtol=1e-8,
                                          max_cycles=60, mixed=mixed, arrival_time=float(arrivals[i])))
                    i += 1
                run_, q = srv.step()
                if i >= nreq and run_ == 0 and q == 0:
                    break
        t1 = srv.now()
        sts = [srv.status(j) for j in ids]
        srv.close()
        lat = np.array([s["t_done"] - s["t_arrival"] for s in sts])
        ok = sum(1 for s in sts if s["state"] == H.CONVERGED)
        return {"solves_per_s": nreq / (t1 - t0), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "converged": ok, "seconds": t1 - t0}

    served = run(mixed=True, sequential=False)
    batched = run(mixed=False, sequential=False, width=8)
    warm = run(mixed=False, sequential=True)
    cold = plain(reqs)
    return {"requests": nreq, "distinct_hierarchies": len(keys),
            "sample": "cube L3-7 / shell(ntan=3,nrad=2) L3-5, P1 Poisson 30% / div-k-grad 70%, 2 coefficient phases, "
                      "Poisson arrivals mean 0.5 ms",
            "served_mixed": served, "served_batched_fp64": batched, "batch_width": 8,
            "sequential_plain_fp64": cold, "sequential_warm_fp64": warm,
            "speedup_solves_per_s": served["solves_per_s"] / cold["solves_per_s"],
            "speedup_vs_sequential_warm": served["solves_per_s"] / warm["solves_per_s"],
            "speedup_batched_vs_sequential_warm": batched["solves_per_s"] / warm["solves_per_s"]}


def stokes_leg(H, ctx, level=3, cycles=3):
    """Configuration 4's system at a reduced level: P2-P1 Taylor-Hood Stokes on the blended shell
    ntan=5, nrad=3 (1920 macro-cells), viscosity eta = exp(2.99 (1 - r) / 0.45), buoyancy-like
    right-hand side (seeded uniform [0, 1] times the position vector in the velocity, zero in the
    pressure), Uzawa multigrid (V(3,3) Uzawa steps with Chebyshev(3) velocity smoothing, quadratic /
    linear transfers, 100 Uzawa steps on level 0), FP64.  Times `cycles` V-cycles after two warm-up
    cycles (setup, a first cycle, the capture of the cycle's CUDA graph) and reports the
    residual-reduction factors."""
    pm = H.PrimitiveStorage.spherical_shell(5, 3, 0.55, 1.0, ctx=ctx)
    st = H.StokesUzawaMultigrid(ctx, pm, 0, level, viscosity=("radial", 2.99, 1.0, 0.45), blending="shell")
    u = [H.P2Function("u%d" % k, pm, 0, level, ctx) for k in range(3)]
    p = H.P1Function("p", pm, 0, level, ctx)
    bu = [H.P2Function("bu%d" % k, pm, 0, level, ctx) for k in range(3)]
    bp = H.P1Function("bp", pm, 0, level, ctx)
    T = H.P2Function("T", pm, 0, level, ctx)
    half = H.P2Function("half", pm, 0, level, ctx)
    T.fill_random(level, 11)  # uniform [-1, 1] ...
    half.interpolate(0.5, level)
    T.assign([0.5, 1.0], [T, half], level)  # ... mapped to [0, 1]
    for k in range(3):
        # buoyancy: T x_k / |x| with T in [0, 1]
        bu[k].interpolate(lambda x, y, z, k=k: [x, y, z][k] / max((x * x + y * y + z * z) ** 0.5, 1e-12), level)
        bu[k].multElementwise([bu[k], T], level)
    st.solve(u, p, bu, bp, level, 2)  # setup (radii, stored matrices), a first cycle and the cycle's graph capture
    ctx.synchronize()
    t0 = time.perf_counter()
    hist = st.solve(u, p, bu, bp, level, cycles)
    ctx.synchronize()
    sec = (time.perf_counter() - t0) / cycles
    nu = pm.packed_size(level + 1)
    # time to rtol 1e-6 one level lower: plain FP64 cycles against FP64 defect correction around FP32
    # cycles (the configuration's "FP32 inner / FP64 outer residual")
    Lr = level - 1
    sr = H.StokesUzawaMultigrid(ctx, pm, 0, Lr, viscosity=("radial", 2.99, 1.0, 0.45), blending="shell")
    si = H.StokesUzawaMultigrid(ctx, pm, 0, Lr, viscosity=("radial", 2.99, 1.0, 0.45), blending="shell")
    runs = {}
    for mode in ("fp64", "fp32_inner"):
        uu = [H.P2Function("uu%d" % k, pm, 0, Lr, ctx) for k in range(3)]
        pp = H.P1Function("pp", pm, 0, Lr, ctx)
        bl_ = [H.P2Function("bl%d" % k, pm, 0, Lr, ctx) for k in range(3)]
        bpl = H.P1Function("bpl", pm, 0, Lr, ctx)
        for k in range(3):
            bl_[k].interpolate(lambda x, y, z, k=k: [x, y, z][k] / max((x * x + y * y + z * z) ** 0.5, 1e-12), Lr)
        if mode == "fp64":
            sr.solve(uu, pp, bl_, bpl, Lr, 2)  # setup and graph capture
            for k in range(3):
                uu[k].interpolate(0.0, Lr)
            pp.interpolate(0.0, Lr)
            ctx.synchronize()
            t0 = time.perf_counter()
            h = sr.solve(uu, pp, bl_, bpl, Lr, 150, rtol=1e-6)
        else:
            sr.mixed_solve(si, uu, pp, bl_, bpl, Lr, max_outer=2, rtol=1e-6)  # setup and graph capture of the inner solver
            for k in range(3):
                uu[k].interpolate(0.0, Lr)
            pp.interpolate(0.0, Lr)
            ctx.synchronize()
            t0 = time.perf_counter()
            h = sr.mixed_solve(si, uu, pp, bl_, bpl, Lr, max_outer=150, rtol=1e-6)
        ctx.synchronize()
        runs[mode] = {"seconds": time.perf_counter() - t0, "cycles": len(h) - 1, "rel_residual": float(h[-1] / h[0]),
                      "u": [uu[k].download(Lr) for k in range(3)]}
    ref = runs["fp64"]["u"]
    scale = max(np.abs(r).max() for r in ref)
    for mode in runs:
        runs[mode]["rel_diff_vs_fp64_solution"] = float(max(np.abs(runs[mode]["u"][k] - ref[k]).max() for k in range(3)) / scale)
        del runs[mode]["u"]
    runs["fp32_inner"]["speedup_vs_fp64"] = runs["fp64"]["seconds"] / runs["fp32_inner"]["seconds"]
    # the same system with the full viscous velocity block (strain-rate form, components coupled)
    sv = H.StokesUzawaMultigrid(ctx, pm, 0, level, viscosity=("radial", 2.99, 1.0, 0.45), blending="shell",
                                velocity_block="full_viscous")
    for k in range(3):
        u[k].interpolate(0.0, level)
    p.interpolate(0.0, level)
    sv.solve(u, p, bu, bp, level, 2)  # setup (radii), a first cycle and the graph capture
    ctx.synchronize()
    t0 = time.perf_counter()
    hv = sv.solve(u, p, bu, bp, level, 2)
    ctx.synchronize()
    full_viscous = {"ms_per_cycle": (time.perf_counter() - t0) / 2 * 1e3, "factors": [float(f) for f in hv[1:] / hv[:-1]],
                    "velocity_block": "2 eta eps(u) : eps(v) - (2/3) eta div u div v, matrix-free, Chebyshev(3) on the coupled block"}
    return {"mesh": "spherical shell ntan=5 nrad=3 (1920 macro-cells), IcosahedralShellMap blending", "level": level,
            "time_to_rtol_1e-6": {"level": Lr, "rhs": "x / |x| (unit buoyancy)", **runs}, "full_viscous": full_viscous,
            "viscosity": "exp(2.99 (1 - r) / 0.45)", "velocity_dofs": 3 * nu, "pressure_dofs": pm.packed_size(level),
            "cycle": "V(3,3) Uzawa (Chebyshev(3) x 3 velocity sweeps, omega 0.7, inverted PSPG diagonal), 30 coarse Uzawa steps",
            "ms_per_cycle": sec * 1e3, "factors": [float(f) for f in hist[1:] / hist[:-1]], "dtype": "f64",
            "stored_velocity_matrices": True}


def p2_leg(H, ctx, level=5, cycle_level=3):
    """Configuration 2's operator: P2 -div(k grad u) with the icosahedral-shell blending map on the
    shell ntan=5, nrad=3 (1920 macro-cells), k = exp(0.5 sin(2 pi x) cos(2 pi y) sin(2 pi z)), FP64.
    Times one apply at `level` (element integrals recomputed every apply, as the reference's
    elementwise operator does) and with stored element matrices one level lower, and one V(3,3)
    Chebyshev(3) cycle on levels 0..cycle_level.  The reference counts 11,678 flops per micro-cell for
    assembling the 10x10 matrix (p2_div_k_grad_blending_q4.hpp:91-98) plus 200 for the matvec; that
    count gives the GFLOP/s figure (this implementation needs fewer: it never forms the matrix)."""
    import torch

    K = ("expsin", 0.5, (0.0, 0.0, 0.0))
    pm = H.PrimitiveStorage.spherical_shell(5, 3, 0.55, 1.0, ctx=ctx)
    nC = pm.counts()[3]

    def time_apply(A, L, reps):
        x = H.P2Function("x", pm, L, L, ctx)
        y = H.P2Function("y", pm, L, L, ctx)
        x.fill_random(L, 1)
        A.apply(x, y, L, H.Inner)
        ctx.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            A.apply(x, y, L, H.Inner)
        ctx.synchronize()
        return (time.perf_counter() - t0) / reps

    out = {"mesh": "spherical shell ntan=5 nrad=3 (1920 macro-cells), IcosahedralShellMap blending",
           "coefficient": "exp(0.5 sin(2 pi x) cos(2 pi y) sin(2 pi z))", "dtype": "f64"}
    A = H.P2ElementwiseBlendingDivKGradOperator(pm, level, level, ctx, k=K, blending="shell")
    sec = time_apply(A, level, 3)
    mc = nC * (1 << level) ** 3
    out["apply"] = {"level": level, "micro_cells": mc, "dofs": pm.packed_size(level + 1), "ms": sec * 1e3,
                    "Mcells_per_s": mc / sec / 1e6, "gflops_reference_count": mc * 11878 / sec / 1e9}
    del A
    # the hyteg-operators form: k stored as a P2 function (interpolated at the blended nodes)
    An = H.P2ElementwiseDivKGradOperator(pm, level, level, ctx, k=K, blending="shell")
    sec = time_apply(An, level, 3)
    out["apply_nodal_coefficient"] = {"level": level, "micro_cells": mc, "ms": sec * 1e3, "Mcells_per_s": mc / sec / 1e6,
                                      "operator": "P2ElementwiseDivKGradIcosahedralShellMap form (k as a P2 function)"}
    del An
    Ls = level - 1
    S = H.P2ElementwiseBlendingDivKGradOperator(pm, Ls, Ls, ctx, k=K, blending="shell")
    S.computeAndStoreLocalElementMatrices()
    sec = time_apply(S, Ls, 5)
    mcs = nC * (1 << Ls) ** 3
    out["apply_stored"] = {"level": Ls, "micro_cells": mcs, "ms": sec * 1e3, "Mcells_per_s": mcs / sec / 1e6,
                           "bytes_per_micro_cell": 55 * 8}
    del S
    Ac = H.P2ElementwiseBlendingDivKGradOperator(pm, 0, cycle_level, ctx, k=K, blending="shell")
    Ac.computeAndStoreLocalElementMatrices()
    g = H.GeometricMultigridSolver(ctx, Ac, 0, cycle_level, 3, 3, smoother="chebyshev", chebyshev_order=3,
                                   power_iterations=20)
    x = H.P2Function("xv", pm, 0, cycle_level, ctx)
    b = H.P2Function("bv", pm, 0, cycle_level, ctx)
    b.fill_random(cycle_level, 3)
    hist = g.solve_cycles(x, b, cycle_level, 2)  # setup, capture, two cycles
    ctx.synchronize()
    t0 = time.perf_counter()
    n = 3
    for _ in range(n):
        g.solve(Ac, x, b, cycle_level)
    ctx.synchronize()
    out["vcycle"] = {"levels": f"0..{cycle_level}", "ms_per_cycle": (time.perf_counter() - t0) / n * 1e3,
                     "cycle": "V(3,3) Chebyshev(3), stored element matrices, CG coarse", "factors": list(hist[1:] / hist[:-1])}
    return out


def p2_constant_leg(H, ctx, level=7, cycle_level=7):
    """P2 constant-stencil Laplacian (P2ConstantLaplaceOperator) on the six-tetrahedra cube at P2 level 7
    (its nodes are the level-8 grid: 16,974,593 DoFs, 16,581,375 inner), FP64: one apply timed with CUDA
    events (algorithmic bytes: read x, write y per inner DoF, 16 B), and one V(3,3) Chebyshev(3) cycle
    with quadratic transfers on levels 0..cycle_level (graph-captured)."""
    import torch

    pm = H.PrimitiveStorage.cuboid(ctx=ctx)
    A = H.P2ConstantLaplaceOperator(pm, 0, level, ctx)
    x = H.P2Function("p2x", pm, level, level, ctx)
    y = H.P2Function("p2y", pm, level, level, ctx)
    x.fill_random(level, 11)
    for _ in range(3):
        A.apply(x, y, level, H.Inner)
    ctx.synchronize()
    s = torch.cuda.ExternalStream(ctx.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    e0.record(s)
    for _ in range(reps):
        A.apply(x, y, level, H.Inner)
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    ndof = inner_dofs(level + 1)
    peak, peak_kind = measured_peak()
    achieved = 16 * ndof / (ms * 1e-3) / 1e9
    out = {"mesh": "unit cube, 6 macro-tets", "level": level, "inner_dofs": ndof, "dtype": "f64",
           "apply_ms": ms, "mdofs": ndof / (ms * 1e-3) / 1e6,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_kind": peak_kind, "kernel": "k_p2c_sweep<double,double,OP_APPLY> + k_p2c_bnd"}}
    del x, y
    g = H.GeometricMultigridSolver(ctx, A, 0, cycle_level, 3, 3, smoother="chebyshev", chebyshev_order=3,
                                   power_iterations=20)
    xv = H.P2Function("p2xv", pm, 0, cycle_level, ctx)
    bv = H.P2Function("p2bv", pm, 0, cycle_level, ctx)
    bv.fill_random(cycle_level, 3)
    hist = g.solve_cycles(xv, bv, cycle_level, 2)  # set-up, capture, two cycles
    ctx.synchronize()
    v0, v1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    v0.record(s)
    n = 3
    for _ in range(n):
        g.solve(A, xv, bv, cycle_level)
    v1.record(s)
    v1.synchronize()
    out["vcycle"] = {"levels": f"0..{cycle_level}", "ms_per_cycle": v0.elapsed_time(v1) / n,
                     "cycle": "V(3,3) Chebyshev(3), quadratic transfers, CG coarse",
                     "factors": [float(f) for f in hist[1:] / hist[:-1]]}
    return out


def config2_solve(H, rtol=1e-10, level=6, max_cycles=40):
    """Configuration 2 as stated: -div(k grad u) = f, P2 elementwise operator with the form
    p2_div_k_grad_blending_q4 (matrix-free: the level-6 element matrices would need 221 GB), thick
    spherical shell r in [0.55, 1] (ntan 5, nrad 3, 1920 macro-cells) with the icosahedral shell map,
    k = exp(0.5 sin(2 pi x) cos(2 pi y) sin(2 pi z)), rhs seeded uniform [-1, 1] on inner DoFs, zero
    guess, V(3,3) with Chebyshev(3) smoothing (spectral radii by 20 power iterations per level), CG coarse
    solve on level 0, FP64, to ||r||/||r0|| <= 1e-10.  Times set-up and the solve separately with CUDA events."""
    import torch

    ctx = H.Context(0)
    s = torch.cuda.ExternalStream(ctx.stream)
    K = ("expsin", 0.5, (0.0, 0.0, 0.0))
    pm = H.PrimitiveStorage.spherical_shell(5, 3, 0.55, 1.0, ctx=ctx)
    A = H.P2ElementwiseBlendingDivKGradOperator(pm, 0, level, ctx, k=K, blending="shell")
    x = H.P2Function("x", pm, 0, level, ctx)
    b = H.P2Function("b", pm, 0, level, ctx)
    b.fill_random(level, 2026)
    b.interpolate(0.0, level, H.DirichletBoundary)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record(s)
    g = H.GeometricMultigridSolver(ctx, A, 0, level, 3, 3, smoother="chebyshev", chebyshev_order=3, power_iterations=20)
    g.smooth(x, b, level, 0)  # set-up: inverse diagonals, spectral radii, coarse CG probe
    e[1].record(s)
    hist = g.solve_cycles(x, b, level, max_cycles, rtol=rtol)
    e[2].record(s)
    e[2].synchronize()
    setup_s, solve_s = e[0].elapsed_time(e[1]) / 1e3, e[1].elapsed_time(e[2]) / 1e3
    f = hist[1:] / hist[:-1]
    return {"config": "configuration 2: P2 div-k-grad, shell (5,3) with IcosahedralShellMap, level 6, FP64",
            "dofs": pm.packed_size(level + 1), "micro_cells": pm.counts()[3] * (1 << level) ** 3,
            "rtol": rtol, "cycles": int(hist.size - 1), "rel_residual": float(hist[-1] / hist[0]),
            "factors": [float(v) for v in f], "setup_s": setup_s, "solve_s": solve_s,
            "s_per_cycle": solve_s / max(1, hist.size - 1),
            "cycle": "V(3,3) Chebyshev(3), matrix-free elementwise apply, CG coarse level 0", "rhs": "seeded uniform [-1,1]"}


def config4_solve(H, rtol=1e-8, level=5, max_outer=60):
    """Configuration 4 as stated: Stokes P2-P1 Taylor-Hood on the shell (5,3) with the icosahedral shell
    map, level 5, viscosity eta = exp(2.99 (1 - r) / 0.45), buoyancy rhs T r/|r| with T seeded uniform in
    [0, 1] (velocity), zero pressure rhs, Uzawa multigrid V(3,3) (Chebyshev(3) velocity sweeps, pressure
    update scaled by the inverse lumped pressure mass weighted by 1/eta, omega = 1/rho from the relaxation
    estimate: 20 power iterations with two velocity sweeps on level 2, as the reference's apps call
    estimateUzawaRelaxationParameter), FP32 inner cycles inside FP64 defect correction to ||r||/||r0|| <=
    1e-8, and the plain FP64 cycles for comparison.  CUDA-event timing of set-up and solve."""
    import torch

    ctx = H.Context(0)
    s = torch.cuda.ExternalStream(ctx.stream)
    pm = H.PrimitiveStorage.spherical_shell(5, 3, 0.55, 1.0, ctx=ctx)
    visc = ("radial", 2.99, 1.0, 0.45)
    u = [H.P2Function("u%d" % k, pm, 0, level, ctx) for k in range(3)]
    p = H.P1Function("p", pm, 0, level, ctx)
    bu = [H.P2Function("bu%d" % k, pm, 0, level, ctx) for k in range(3)]
    bp = H.P1Function("bp", pm, 0, level, ctx)
    T = H.P2Function("T", pm, level, level, ctx)
    half = H.P2Function("half", pm, level, level, ctx)
    T.fill_random(level, 4)  # uniform [-1, 1] ...
    half.interpolate(0.5, level)
    T.assign([0.5, 1.0], [T, half], level)  # ... mapped to [0, 1]
    for k in range(3):
        bu[k].interpolate(lambda x, y, z, k=k: [x, y, z][k] / max((x * x + y * y + z * z) ** 0.5, 1e-12), level)
        bu[k].multElementwise([bu[k], T], level)
    del T, half
    out = {"config": "configuration 4: Stokes P2-P1, shell (5,3) with IcosahedralShellMap, level 5",
           "velocity_dofs": 3 * pm.packed_size(level + 1), "pressure_dofs": pm.packed_size(level), "rtol": rtol,
           "viscosity": "exp(2.99 (1 - r) / 0.45)", "rhs": "T r/|r|, T seeded uniform [0, 1]",
           "cycle": "V(3,3) Uzawa, Chebyshev(3) x 3 velocity sweeps, pressure update by the inverse lumped mass "
                    "weighted by 1/eta, omega = 1/rho (estimated), 30 coarse Uzawa steps"}
    runs = {}
    for mode in ("fp32_inner_fp64_outer", "fp64"):
        st = H.StokesUzawaMultigrid(ctx, pm, 0, level, viscosity=visc, blending="shell", pressure_scaling="lumped_mass")
        rho = st.estimate_relaxation(2, 20, 2)
        st.set_omega(1.0 / rho)
        out["relaxation_estimate"] = {"level": 2, "power_iterations": 20, "velocity_sweeps": 2, "rho": rho, "omega": 1.0 / rho}
        si = None
        if mode != "fp64":
            si = H.StokesUzawaMultigrid(ctx, pm, 0, level, viscosity=visc, blending="shell", pressure_scaling="lumped_mass")
            si.set_omega(1.0 / rho)
        for rep in range(2):  # the first run sets up (radii, stored matrices, graph capture)
            for k in range(3):
                u[k].interpolate(0.0, level)
            p.interpolate(0.0, level)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            if mode == "fp64":
                h = st.solve(u, p, bu, bp, level, max_outer if rep else 1, rtol=rtol)
            else:
                h = st.mixed_solve(si, u, p, bu, bp, level, max_outer=max_outer if rep else 1, rtol=rtol)
            e1.record(s)
            e1.synchronize()
            if rep == 0:
                setup_s = e0.elapsed_time(e1) / 1e3
        sol = [u[k].download(level) for k in range(3)]
        runs[mode] = {"setup_and_first_cycle_s": setup_s, "solve_s": e0.elapsed_time(e1) / 1e3, "cycles": int(len(h) - 1),
                      "rel_residual": float(h[-1] / h[0]), "factors": [float(f) for f in h[1:] / h[:-1]], "_u": sol}
        del st, si
    ref = runs["fp64"]["_u"]
    scale = max(np.abs(r).max() for r in ref)
    for mode in runs:
        runs[mode]["rel_diff_vs_fp64_solution"] = float(max(np.abs(runs[mode]["_u"][k] - ref[k]).max() for k in range(3)) / scale)
        del runs[mode]["_u"]
    runs["fp32_inner_fp64_outer"]["speedup_vs_fp64"] = runs["fp64"]["solve_s"] / runs["fp32_inner_fp64_outer"]["solve_s"]
    out["runs"] = runs
    return out


def config5_serving(H, nreq=2000, seed=5, rate_hz=400.0, plain_sample=40):
    """Configuration 5 as stated: a stream of 2000 solve requests with Poisson arrivals (seeded, mean rate
    400/s, above what one GPU sustains), each a P1 or P2 diffusion solve (-div(k grad u), k = exp(0.5
    sin cos sin) with one of four phases) on the six-tetrahedra cube or the icosahedral shell with ntan in
    {3, 5} and nrad 3 (shell blending; the classic shell mesh needs ntan - 1 a power of two, which leaves
    3 and 5 of the range 3-5), level uniform in 3..7, rtol 1e-8.  P1 requests run FP64 defect
    correction around FP32 cycles; P2 requests run FP64 cycles (the loop's defect correction is written
    for P1); both on resident one-solve slots with graph-captured cycles.  Requests whose hierarchy can
    never fit the HBM budget are rejected at submission and counted.  Reports solves/s, p50/p99 latency
    (arrival to solution) and the rejected count; no set-up is done before the clock starts.  Baseline:
    sequential plain FP64 solves through the plain drop-in API (operator with stored matrices, solver,
    functions built per request, solution read back) on a seeded sample of `plain_sample` admitted
    requests, its solves/s taken as the sample's count over its time."""
    import torch

    ctx = H.Context(0)
    rng = np.random.default_rng(seed)
    meshes = {"cube": H.PrimitiveStorage.cuboid(ctx=ctx)}
    for nt in (3, 5):
        meshes[f"shell{nt}"] = H.PrimitiveStorage.spherical_shell(nt, 3, 0.55, 1.0, ctx=ctx)
    phases = [(0.0, 0.0, 0.0), (0.13, 0.27, 0.41), (0.71, 0.05, 0.33), (0.29, 0.83, 0.61)]
    reqs = []
    for i in range(nreq):
        m = ["cube", "shell3", "shell5"][int(rng.integers(0, 3))]
        p2 = bool(rng.random() < 0.5)
        L = int(rng.integers(3, 8))
        ph = phases[int(rng.integers(0, 4))]
        reqs.append((m, L, "p2_divkgrad" if p2 else "divkgrad", ("expsin", 0.5, ph), "shell" if m != "cube" else None,
                     int(rng.integers(1, 2**31)), not p2))
    free0, total = torch.cuda.mem_get_info()
    budget = 0.6 * free0  # admission budget, with room for the meshes' level tables and estimate error
    srv = H.SolveServer(ctx, max_slots=64, hbm_budget_bytes=budget)
    arrivals = srv.now() + np.cumsum(rng.exponential(1.0 / rate_hz, nreq))
    min_free = free0
    ids, admitted, rejected, i = [], [], 0, 0
    t0 = srv.now()
    while True:
        now = srv.now()
        while i < nreq and arrivals[i] <= now:
            r = reqs[i]
            try:
                ids.append(srv.submit(meshes[r[0]], r[1], kind=r[2], k=r[3], blending=r[4], seed=r[5], rtol=1e-8, max_cycles=60,
                                      mixed=r[6], arrival_time=float(arrivals[i])))
                admitted.append(r)
            except H.HybError:
                rejected += 1
            i += 1
        run_, q = srv.step()
        min_free = min(min_free, torch.cuda.mem_get_info()[0])
        if i >= nreq and run_ == 0 and q == 0:
            break
    t1 = srv.now()
    sts = [srv.status(j) for j in ids]
    srv.close()
    done = [s for s in sts if s["state"] == H.CONVERGED]
    lat = np.array([s["t_done"] - s["t_arrival"] for s in done])
    # time in service (admission to solution) per request class; solves overlap, so the sums exceed
    # the stream's wall time
    classes = {}
    for r, st in zip(admitted, sts):
        c = classes.setdefault(f"{r[2]} {r[0]} L{r[1]}", {"n": 0, "service_s": 0.0, "cycles": 0})
        c["n"] += 1
        c["service_s"] += max(0.0, st["t_done"] - st["t_admit"])
        c["cycles"] += st["cycles"]
    rejected_classes = sorted(set(f"{r[2]} {r[0]} L{r[1]}" for r in reqs[:i] if r not in admitted))
    out = {"config": "configuration 5: serving stream", "requests": nreq, "admitted": len(ids), "rejected_hbm": rejected,
           "converged": len(done), "seconds": t1 - t0, "solves_per_s": len(done) / (t1 - t0),
           "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
           "cycles_mean": float(np.mean([s["cycles"] for s in done])),
           "hbm_budget_gb": budget / 1e9, "peak_device_use_gb": (total - min_free) / 1e9,
           "service_by_class": dict(sorted(classes.items(), key=lambda kv: -kv[1]["service_s"])[:12]),
           "rejected_classes": rejected_classes,
           "mix": "P1 (FP32 inner / FP64 outer) or P2 (FP64); cube or shell ntan 3/5 nrad 3; levels 3-7; "
                  "k = exp(0.5 sin cos sin), 4 phases; Poisson arrivals 400/s"}
    # sequential plain FP64 solves of a seeded sample of the admitted requests
    pick = np.random.default_rng(seed + 1).choice(len(admitted), size=min(plain_sample, len(admitted)), replace=False)
    tp0, okp = time.perf_counter(), 0
    for j in sorted(pick):
        m, L, kind, kk, bl, sd, _ = admitted[j]
        pm = meshes[m]
        if kind == "p2_divkgrad":
            A = H.P2ElementwiseBlendingDivKGradOperator(pm, 0, L, ctx, k=kk, blending=bl)
            x, b = H.P2Function("x", pm, 0, L, ctx), H.P2Function("b", pm, 0, L, ctx)
        else:
            A = H.P1ElementwiseBlendingDivKGradOperator(pm, 0, L, ctx, k=kk, blending=bl)
            x, b = H.P1Function("x", pm, 0, L, ctx), H.P1Function("b", pm, 0, L, ctx)
        A.computeAndStoreLocalElementMatrices()
        g = H.GeometricMultigridSolver(ctx, A, 0, L, 3, 3, smoother="chebyshev", chebyshev_order=3, power_iterations=20)
        b.fill_random(L, sd)
        hist = g.solve_cycles(x, b, L, 60, rtol=1e-8)
        x.download(L)
        okp += int(hist[-1] < 1e-8 * hist[0])
        g.close()
        del A, g, x, b
    tp = time.perf_counter() - tp0
    out["sequential_plain_fp64_sample"] = {"requests": len(pick), "converged": okp, "seconds": tp,
                                           "solves_per_s": len(pick) / tp}
    out["speedup_vs_sequential_plain_fp64"] = out["solves_per_s"] / out["sequential_plain_fp64_sample"]["solves_per_s"]
    return out


def p2_cpu_reference(cells=400000):
    """The reference's per-micro-cell work of the P2 elementwise apply (integrateAll of the generated
    form + 10x10 matvec), compiled from its sources, on the host cores (test blending map)."""
    import ctypes as C

    from oracle import ref as R

    if not R.available():
        return None
    f = R.lib().ref_p2_elem_apply_bench
    f.restype, f.argtypes = C.c_double, [C.c_long, C.c_int, C.c_double]
    threads = os.cpu_count() or 1
    sec = f(cells, threads, 0.5)
    return {"Mcells_per_s": cells / sec / 1e6, "cores": threads, "kind": "reference",
            "sample": f"{cells} micro-cells of p2_div_k_grad_blending_q4 integrateAll + matvec, OpenMP"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    L = args.level
    n = 1 << L
    from oracle import hyteg_oracle as O
    from oracle import ref as R

    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libhyteg_ref.so was not built"}))
        return
    for _ in range(args.warmup):
        cpu_reference_apply(L, max_steps=1)
    rate, k, threads, el = cpu_reference_apply(L, max_steps=args.steps)
    cell_inner = 6 * O.tet_size(n - 3)
    ms = el / k * 1e3
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world, "steps": k,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded uniform [-1,1] input)",
        "config": {"workload": WORKLOAD + " (macro-cell interiors, the reference's generated kernel)", "level": L,
                   "inner_dofs_cells": cell_inner},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{k} full applies of the 6 macro-cell interiors at level {L}"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def profile_vcycle(args):
    """One FP64 and one FP32-storage V(3,3) Chebyshev(3) cycle on the six-tetrahedra cube at the bench
    level, launched kernel by kernel (no graph), each inside cudaProfilerStart/Stop after a setup
    cycle; prints the wall time per cycle of three uncaptured cycles per value type."""
    import torch

    import hyteg_b200 as H

    ctx = H.Context(0)
    pm = H.PrimitiveStorage.cuboid(ctx=ctx)
    L = args.level
    A = H.P1ConstantLaplaceOperator(pm, 0, L, ctx)
    out = {}
    for dt in ("float64", "float32"):
        x = H.P1Function("x", pm, 0, L, ctx, dtype=dt)
        b = H.P1Function("b", pm, 0, L, ctx, dtype=dt)
        b.fill_random(L, 5)
        g = H.GeometricMultigridSolver(ctx, A, 0, L, 3, 3, smoother="chebyshev", chebyshev_order=3, power_iterations=20,
                                       use_graph=False)
        g.solve(A, x, b, L)  # setup
        ctx.synchronize()
        t0 = time.perf_counter()
        for _ in range(3):
            g.solve(A, x, b, L)
        ctx.synchronize()
        out[dt] = (time.perf_counter() - t0) / 3 * 1e3
        torch.cuda.profiler.start()
        g.solve(A, x, b, L)
        ctx.synchronize()
        torch.cuda.profiler.stop()
    print(json.dumps({"profile_vcycle_ms_per_cycle_without_graph": out, "level": L}))


def run_ours(args, rank, world, local):
    import torch

    import hyteg_b200 as H

    if args.profile_vcycle:
        return profile_vcycle(args)
    if args.config2:
        print(json.dumps(config2_solve(H)))
        return
    if args.config4:
        print(json.dumps(config4_solve(H)))
        return
    if args.config5:
        print(json.dumps(config5_serving(H, nreq=args.config5_requests)))
        return

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    L = args.level
    ctx = H.Context(local, stream.cuda_stream)
    pm = H.PrimitiveStorage.cuboid(ctx=ctx)
    A = H.P1ConstantLaplaceOperator(pm, 0, L, ctx)
    x = H.P1Function("x", pm, L, L, ctx)
    y = H.P1Function("y", pm, L, L, ctx)
    packed = pm.packed_size(L)
    rng = np.random.default_rng(1234 + rank)
    host_x = rng.uniform(-1.0, 1.0, packed)
    x.upload(L, host_x)
    ndof = inner_dofs(L)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # device-resident timing (inputs in HBM; each 136 MB vector exceeds the 126 MB L2)
    for _ in range(max(3, args.warmup)):
        A.apply(x, y, L, H.Inner)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    l0 = ctx.launches
    with torch.cuda.stream(stream):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            e0.record(stream)
            for _ in range(args.steps):
                A.apply(x, y, L, H.Inner)
            e1.record(stream)
            e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    launches = ctx.launches - l0
    barrier()
    torch.cuda.synchronize()
    ms_max, value = job_rate(ms, ndof, world, "cuda")

    # end to end through the public API: host vector in (pinned host memory), apply, host vector out
    # (pinned); each transfer is one contiguous copy plus a device repack
    e2e_steps = max(3, min(args.steps, 10))
    pin_x = torch.empty(packed, dtype=torch.float64, pin_memory=True).numpy()
    pin_y = torch.empty(packed, dtype=torch.float64, pin_memory=True).numpy()
    pin_x[:] = host_x
    x.upload(L, pin_x)
    y.download(L, out=pin_y)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        x.upload(L, pin_x)
        A.apply(x, y, L, H.Inner)
        out = y.download(L, out=pin_y)
    t_serial = (time.perf_counter() - t0) / e2e_steps
    # the same steps double-buffered: step s runs on context s % 2 (own stream, own operator, own
    # vectors and staging), so the host-to-device copy of one step overlaps the device-to-host copy of
    # the other through the two copy directions; every step still moves its whole input and output
    ectx = [H.Context(local), H.Context(local)]
    eA = [H.P1ConstantLaplaceOperator(pm, L, L, c) for c in ectx]
    ex = [H.P1Function("ex%d" % i, pm, L, L, c) for i, c in enumerate(ectx)]
    ey = [H.P1Function("ey%d" % i, pm, L, L, c) for i, c in enumerate(ectx)]
    px = [pin_x, torch.empty(packed, dtype=torch.float64, pin_memory=True).numpy()]
    px[1][:] = host_x
    py = [pin_y, torch.empty(packed, dtype=torch.float64, pin_memory=True).numpy()]
    for i in range(2):
        ex[i].upload_async(L, px[i])
        eA[i].apply(ex[i], ey[i], L, H.Inner)
        ey[i].download_async(L, py[i])
    for c in ectx:
        c.synchronize()
    t0 = time.perf_counter()
    for s_ in range(e2e_steps):
        i = s_ % 2
        ex[i].upload_async(L, px[i])
        eA[i].apply(ex[i], ey[i], L, H.Inner)
        ey[i].download_async(L, py[i])
    for c in ectx:
        c.synchronize()
    t_e2e = (time.perf_counter() - t0) / e2e_steps
    assert np.array_equal(py[0], py[1]) and np.array_equal(py[0], out)
    _, e2e_value = job_rate(t_e2e * 1e3, ndof, world, "cuda")

    # one FP64 V(3,3) Chebyshev(3) multigrid cycle on the same level (graph-captured)
    vcycle = None
    if not args.no_vcycle:
        b = H.P1Function("b", pm, 0, L, ctx)
        xv = H.P1Function("xv", pm, 0, L, ctx)
        b.upload(L, np.where(np.abs(host_x) > 0, rng.uniform(-1, 1, packed), 0.0))
        gmg = H.GeometricMultigridSolver(ctx, A, 0, L, preSmoothSteps=3, postSmoothSteps=3, smoother="chebyshev",
                                         chebyshev_order=3, power_iterations=20)
        gmg.solve(A, xv, b, L)  # setup + capture
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            v0 = torch.cuda.Event(enable_timing=True)
            v1 = torch.cuda.Event(enable_timing=True)
            v0.record(stream)
            nv = 5
            for _ in range(nv):
                gmg.solve(A, xv, b, L)
            v1.record(stream)
            v1.synchronize()
        vcycle = {"ms_per_cycle": v0.elapsed_time(v1) / nv, "cycle": "V(3,3) Chebyshev(3), CG coarse level 0",
                  "dtype": "f64", "graph": True}

    if rank != 0:
        return
    A.apply(x, y, L, H.Inner)
    parity = reference_parity(H, pm, x, y, L)
    config1 = None if args.no_config1 else config1_leg(H, ctx)
    p2c = None if args.no_p2c else p2_constant_leg(H, ctx)
    mixed = None if args.no_mixed else mixed_precision_leg(H, ctx, pm, A, L)
    serving = None if args.no_serve else serving_leg(H, ctx, nreq=args.serve_requests)
    p2 = None
    if not args.no_p2:
        p2 = p2_leg(H, ctx)
        p2["cpu_baseline"] = p2_cpu_reference()
    stokes = None
    if not args.no_stokes:
        stokes = stokes_leg(H, ctx)
    peak, peak_kind = measured_peak()
    alg_bytes = 2 * 8 * ndof  # read x, write y per inner DoF
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    cpu = cpu_reference_apply(L, seconds=10.0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded uniform [-1,1] input vector)",
        "config": {"workload": WORKLOAD, "level": L, "inner_dofs": ndof, "dofs": (2 ** L + 1) ** 3,
                   "l2": "inputs larger than L2 (136 MB per vector)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": profile_traffic(),
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "kernel": "k_cell_sweep<double,double,OP_APPLY> + k_bnd_stencil (one apply)"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": packed * 8, "d2h_bytes_per_step": packed * 8,
                "steps": "double-buffered on two streams (upload, apply, download per step)",
                "serial_value": world * ndof / t_serial / 1e6},
        "gpu_launches": launches,
        "parity_rel_err": parity,
        "parity_check": "cell interiors of the timed apply against the reference's compiled "
                        "apply_3D_macrocell_vertexdof_to_vertexdof_replace on the same input (max norm, relative)",
        "clocks": clk.summary(),
    }
    if vcycle:
        line["vcycle"] = vcycle
    if config1:
        line["config1_poisson_cube_L5"] = config1
    if p2c:
        line["p2_constant_cube"] = p2c
    if mixed:
        line["mixed_precision"] = mixed
    if serving:
        line["serving"] = serving
    if p2:
        line["p2_divkgrad_shell"] = p2
    if stokes:
        line["stokes_shell"] = stokes
    if cpu:
        rate, k, threads, el = cpu
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                                "sample": f"{k} applies of the 6 macro-cell interiors at level {L} in {el:.1f} s "
                                          f"(reference's generated kernel, one macro-cell per thread: {threads} of "
                                          f"{os.cpu_count()} host cores, the reference parallelises applies over macro-cells)"}
    print(json.dumps(line))


def main():
    args = parse()
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
