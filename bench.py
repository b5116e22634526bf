"""Benchmark: NS steps/s of the 4-step projection on the periodic Taylor-Green
vortex, 256x256 Q2 elements (262,144 unique nodes), FP64, multigrid-PCG
pressure (final mesh 4x4, tol 1e-8), BiCGSTAB momentum (tol 1e-8).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). Under torchrun (N > 1) every rank runs an
independent replica of the workload on its own GPU (a single solve does not
shard: replicas only); the step time is the max over ranks.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(workload="taylor_green_periodic_q2_256x256", nex=256, ney=256, order=2, domain="[0,2pi]^2",
                nu=0.01, rho=1.0, dt=1e-3, pressure_precond="multigrid", final_multigrid_mesh=[4, 4],
                solver_tol=1e-8, set_zeroP=False)
STAGES = ["convection_build", "momentum_rhs", "momentum_bicgstab", "u_star", "ppe_rhs", "pressure_pcg",
          "projection"]
REFERENCE_SAMPLE_S = 60.0
KERNEL_OF_STAGE = {"pressure_pcg": "k_cg<1>", "momentum_bicgstab": "k_bicgstab<1,2>", "convection_build": "k_convection"}


def tg_config(sim, n):
    return sim.Config(mesh="simple", solver="standard",
                      mesh_config=sim.SimpleMeshConfig(num_elem=[n, n], domain_size=[2 * np.pi, 2 * np.pi],
                                                       shape_func_ord=2, periodic=True),
                      solver_config=sim.StandardSolverConfig(dirichlet_faces=[], symmetry_faces=[], outlet_faces=[],
                                                             streamline_diff=False, solver_tol=1e-8, set_zeroP=False,
                                                             pressure_precond="multigrid",
                                                             final_multigrid_mesh=[4, 4]))


def tg_initial(node_coords):
    x, y = node_coords[:, 0], node_coords[:, 1]
    U = np.concatenate([np.sin(x) * np.cos(y), -np.cos(x) * np.sin(y)])
    P = 0.25 * (np.cos(2 * x) + np.cos(2 * y))
    return U, P - P.mean()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback (MEASURED_PEAKS.json absent: 6.65 TB/s, an earlier copy measurement on B200)"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms during the timed
    region: sampling is live before the region starts (the first sample is
    waited for), and only the samples taken after that one are summarised."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")
        self.skip = 0

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            t0 = time.time()
            while time.time() - t0 < 5.0 and self.proc.poll() is None:
                with open(self.path) as g:
                    n = sum(1 for r in g if r.strip())
                if n:
                    self.skip = n
                    break
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        rows = rows[self.skip:] or rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip().lower() == "active"})
        load = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def cg_algorithmic_bytes(level_nn, iters, block_from):
    """Algorithmic DRAM bytes of one k_cg launch (MG-PCG, mean-zero). Per phase:
    the nn-length vectors it must read and write once (FP64), stencil re-reads
    excluded. Init: b, x0 -> r (+centred rhs copy): 5 nn. Per iteration: p/Ap
    phase reads z, p_old, writes p_new, Ap (4 nn); x/r update reads x, p, r, Ap,
    diag and writes x, r (7 nn). Per V-cycle level n: pre-smooth+residual
    reads r, diag, writes x, t (4 nn_n); restriction reads t and diag_{n+1},
    writes r_{n+1} (nn_n + 2 nn_{n+1}); prolongation reads x_{n+1}, x, writes
    t (2 nn_n + nn_{n+1}); post-smooth reads t, r, diag, writes x (4 nn_n).
    The V-cycle of the final iteration is skipped (its z is never used)."""
    w = 8
    L = len(level_nn)
    vcyc = 0
    for n in range(L - 1):
        vcyc += 11 * level_nn[n] + 3 * level_nn[n + 1]
    vcyc += 3 * level_nn[-1]
    nn = level_nn[0]
    total = 5 * nn + vcyc + iters * (11 * nn) + max(iters - 1, 0) * vcyc + 2 * nn
    return total * w


def bicgstab_algorithmic_bytes(nn, ne, nen, ndim, iters, nq=9):
    """k_bicgstab with the on-the-fly convection operator: each operator apply
    reads the Gauss-point factors of Ce(U_n) (3 nq per element, instead of Ce's
    nen^2) plus the vectors of its phase; 3 phases per iteration (see the
    kernel): apply on p (reads r, p_old, q_old, rhat; writes p, q), apply on s
    (reads r, q; writes t), update (reads x, p, r, q, t, rhat; writes x, r)."""
    w = 8
    vec = ndim * nn
    fac = 3 * nq * ne
    init = fac + 6 * vec
    per_it = (fac + 6 * vec) + (fac + 3 * vec) + 8 * vec
    return (init + iters * per_it) * w


def run_ours(args, rank, world, local_rank):
    import torch

    import jax_fem_cfd_b200 as fem
    import jax_fem_cfd_b200.setup.simulation as sim
    from jax_fem_cfd_b200 import _lib

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.size
    compute, timestep, nc, sn, h, nn, gd, Ud = sim.setup(tg_config(sim, n))
    solver = timestep.solver
    ctx = solver.ctx
    U0, P0 = tg_initial(nc.cpu().numpy())
    dt, rho, mu = 1e-3, 1.0, 0.01
    U = torch.as_tensor(U0, device=dev)
    P = torch.as_tensor(P0, device=dev)
    Fp, F = compute(Ud, None, 0.0, dt)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2
    _lib.call("fem_ctx_enable_timing", ctx.handle, 1)
    for _ in range(args.warmup):
        U, P, ui, pi = timestep(U, P, dt, rho, mu, Ud, Fp, F)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stage_ms = np.zeros(len(STAGES))
    iters = []
    barrier(world)
    torch.cuda.synchronize()
    launches0 = _lib.launch_count()
    with ClockSampler(local_rank) as clk:
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            U, P, ui, pi = timestep(U, P, dt, rho, mu, Ud, Fp, F)
            ends[k].record(stream)
            st = (ctypes.c_float * 16)()
            nst = _lib.load().fem_ctx_stage_times(ctx.handle, st, 16)
            stage_ms[:nst] += np.array(st[:nst])
            iters.append((int(ui), int(pi)))
        torch.cuda.synchronize()
    launches = _lib.launch_count() - launches0
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(step_ms))
    total_ms = max_over_ranks(total_ms, world)
    # --- end to end through the public API with host buffers ---
    U_h = torch.as_tensor(U0).pin_memory()
    P_h = torch.as_tensor(P0).pin_memory()
    Uo_h = torch.empty_like(U_h).pin_memory()
    Po_h = torch.empty_like(P_h).pin_memory()
    e_s = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e_e = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    _lib.call("fem_ctx_enable_timing", ctx.handle, 0)
    for k in range(min(args.warmup, 2)):
        Ug, Pg = U_h.to(dev, non_blocking=True), P_h.to(dev, non_blocking=True)
        Fp, F = compute(Ud, None, 0.0, dt)
        Ug, Pg, _, _ = timestep(Ug, Pg, dt, rho, mu, Ud, Fp, F)
        Uo_h.copy_(Ug, non_blocking=True)
        Po_h.copy_(Pg, non_blocking=True)
    torch.cuda.synchronize()
    barrier(world)
    for k in range(args.steps):
        flush.zero_()
        e_s[k].record(stream)
        Ug, Pg = U_h.to(dev, non_blocking=True), P_h.to(dev, non_blocking=True)
        Fp, F = compute(Ud, None, k * dt, (k + 1) * dt)
        Ug, Pg, _, _ = timestep(Ug, Pg, dt, rho, mu, Ud, Fp, F)
        Uo_h.copy_(Ug, non_blocking=True)
        Po_h.copy_(Pg, non_blocking=True)
        e_e[k].record(stream)
        U_h, Uo_h = Uo_h, U_h
        P_h, Po_h = Po_h, P_h
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(float(sum(s.elapsed_time(e) for s, e in zip(e_s, e_e))), world)
    h2d = (U0.size + P0.size) * 8
    d2h = h2d
    res = dict(total_ms=total_ms, step_ms=step_ms, stage_ms=(stage_ms / args.steps).tolist(), iters=iters,
               launches=launches, clocks=clk.summary(), e2e_ms=e2e_ms, h2d=h2d, d2h=d2h, nn=nn, ctx=ctx,
               level_nn=[ctx.level_info(l)[0] for l in range(ctx.nlev)], block_from=None,
               final=(U.clone(), P.clone()), coords=nc)
    return res


def _mixed_inner():
    """FP32 inner iterations per FP64 refinement cycle of StandardSolverConfig(precision="mixed")."""
    from jax_fem_cfd_b200.solvers import standard
    return standard.MIXED_INNER


def tg_mixed(args, fp64_final, coords):
    """The same Taylor-Green workload in mixed precision
    (StandardSolverConfig(precision="mixed"): both solves are FP64 refinement
    to the step's 1e-8, around FP32 Chebyshev-multigrid PCG iterations for the
    pressure and FP32 BiCGSTAB iterations for the momentum):
    warm-up + timed steps exactly as the FP64 run (L2 flushed between timed
    steps, CUDA events), then the final state against the FP64 run's after the
    same steps, and both against the analytic decay u0 exp(-2 nu t)."""
    import torch

    import jax_fem_cfd_b200.setup.simulation as sim
    cfg = tg_config(sim, args.size)
    cfg.solver_config.precision = "mixed"
    compute, timestep, nc, sn, h, nn, gd, Ud = sim.setup(cfg)
    U0, P0 = tg_initial(nc.cpu().numpy())
    dt, rho, mu = 1e-3, 1.0, 0.01
    dev = torch.device("cuda", torch.cuda.current_device())
    U, P = torch.as_tensor(U0, device=dev), torch.as_tensor(P0, device=dev)
    Fp, F = compute(Ud, None, 0.0, dt)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        U, P, ui, pi = timestep(U, P, dt, rho, mu, Ud, Fp, F)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ms, cycles = 0.0, []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        U, P, ui, pi = timestep(U, P, dt, rho, mu, Ud, Fp, F)
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        cycles.append(int(pi))
    nsteps = args.warmup + args.steps
    rel = lambda a, b: float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
    Uf, Pf = fp64_final
    Ua = torch.as_tensor(U0, device=dev) * np.exp(-2 * mu * nsteps * dt)
    return {"workload": "the same Taylor-Green workload, mixed-precision pressure and momentum solves",
            "steps_per_s": args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps,
            "pressure_cycles_mean": float(np.mean(cycles)),
            "pressure_solve": f"FP64 refinement to 1e-8, {_mixed_inner()} FP32 Chebyshev-multigrid PCG iterations per cycle",
            "momentum_solve": "FP64 refinement to 1e-8, 3 FP32 BiCGSTAB iterations per cycle (FP32 Gauss factors)",
            "steps_compared": nsteps,
            "rel_err_vs_fp64": {"U": rel(U, Uf), "P": rel(P, Pf)},
            "rel_err_vs_analytic_velocity": {"fp64": rel(Uf, Ua), "mixed": rel(U, Ua)}}


def tg_mixed_long(steps=500, size=256):
    """The Taylor-Green workload over `steps` steps (the config's 500 by
    default) in FP64 and in mixed precision from the same analytic start, each
    at the step's tol 1e-8: steps/s of each (CUDA events per step, L2 flushed
    between steps), the mixed state against the FP64 one after every 100
    steps, and both against the analytic decay."""
    import torch

    import jax_fem_cfd_b200.setup.simulation as sim
    dt, rho, mu = 1e-3, 1.0, 0.01
    dev = torch.device("cuda", torch.cuda.current_device())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    runs = {}
    for prec in ("fp64", "mixed"):
        cfg = tg_config(sim, size)
        cfg.solver_config.precision = prec
        compute, timestep, nc, sn, h, nn, gd, Ud = sim.setup(cfg)
        U0, P0 = tg_initial(nc.cpu().numpy())
        U, P = torch.as_tensor(U0, device=dev), torch.as_tensor(P0, device=dev)
        Fp, F = compute(Ud, None, 0.0, dt)
        ms, snaps = 0.0, []
        for k in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            U, P, ui, pi = timestep(U, P, dt, rho, mu, Ud, Fp, F)
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            if (k + 1) % 100 == 0 or k + 1 == steps:
                snaps.append((k + 1, U.clone(), P.clone()))
        runs[prec] = (steps / (ms * 1e-3), snaps, U0)
    rel = lambda a, b: float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
    (v64, s64, U0), (vmx, smx, _) = runs["fp64"], runs["mixed"]
    errs = {str(k): {"U": rel(Um, Uf), "P": rel(Pm, Pf)} for (k, Uf, Pf), (_, Um, Pm) in zip(s64, smx)}
    Ua = torch.as_tensor(U0, device=dev) * np.exp(-2 * mu * steps * dt)
    return {"workload": f"Taylor-Green {size}x{size} Q2 periodic, nu 0.01, dt 1e-3, {steps} steps, tol 1e-8",
            "fp64_steps_per_s": v64, "mixed_steps_per_s": vmx, "mixed_speedup": vmx / v64,
            "mixed_rel_err_vs_fp64_by_step": errs,
            "rel_err_vs_analytic_velocity": {"fp64": rel(s64[-1][1], Ua), "mixed": rel(smx[-1][1], Ua)}}


def _dist_device():
    """Device of the collectives' tensors: CUDA under NCCL, host under gloo."""
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.ones(1, device=_dist_device())
        dist.all_reduce(t)
        if t.is_cuda:
            torch.cuda.synchronize()


def max_over_ranks(v, world):
    """Max of a per-rank device time over all ranks (the slowest replica)."""
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=_dist_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, steps, max_total_ms):
    """Whole-job steps/s: every replica advances `steps` steps; the job takes the
    slowest rank's time."""
    return world * 1000.0 * steps / max_total_ms


def poisson(n, solves=5):
    """MG-PCG Poisson solve on an n x n Q1 unit square: pinned node 0, seeded
    random rhs, x0 = 0, tol 1e-8, final MG mesh 4x4. Median of `solves` timed
    solves after 3 warm-up solves, a 256 MiB L2 flush before each. The same for
    the mixed-precision solve (fem_pressure_solve_mixed, same tolerance on the
    FP64 residual); errors of both against an FP64 solve to 1e-12."""
    import torch

    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import Context, Mesh, make_mask, ptr, stream
    from jax_fem_cfd_b200.core import multigrid as mg
    hbm, _ = measured_peaks()
    ctx = Context(Mesh(0, False, n, n, 1, 1.0, 1.0))
    pm = make_mask(np.array([0]), ctx.nn)
    ctx.set_bc(None, pm, True)
    nlev = int(np.log2(n // 4)) + 1
    mg.Hierarchy(ctx, nlev, [np.array([0])] * nlev, 1e-8)
    rng = np.random.default_rng(0)
    b = torch.as_tensor(rng.standard_normal(ctx.nn), device="cuda")
    b[0] = 0.0
    x = torch.zeros_like(b)
    it = torch.zeros(1, dtype=torch.int32, device="cuda")
    stt = torch.zeros(1, dtype=torch.int32, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    times = []
    for k in range(3 + solves):
        x.zero_()
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        _lib.call("fem_pressure_solve", ctx.handle, ptr(b), ptr(x), 1e-8, 0.0, 1000, 4, 0, 1, ptr(it), ptr(stt),
                  stream())
        e.record()
        torch.cuda.synchronize()
        if k >= 3:
            times.append(s.elapsed_time(e))
    ms = float(np.median(times))
    iters = int(it.item())
    status = int(stt.item())
    x64 = x.clone()
    byts = cg_algorithmic_bytes([ctx.level_info(l)[0] for l in range(ctx.nlev)], iters, None)
    # reference solution for the error figures: FP64 MG-PCG to 1e-12 (untimed)
    xr = torch.zeros_like(b)
    _lib.call("fem_pressure_solve", ctx.handle, ptr(b), ptr(xr), 1e-12, 0.0, 1000, 4, 0, 1, ptr(it), ptr(stt),
              stream())
    # mixed precision: FP64 refinement around an FP32 MG-PCG (8 inner iterations), same tolerance
    cyc, res = ctypes.c_int(0), ctypes.c_double(0.0)
    mtimes = []
    for k in range(3 + solves):
        x.zero_()
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        _lib.call("fem_pressure_solve_mixed", ctx.handle, ptr(b), ptr(x), 1e-8, 8, 50, ctypes.byref(cyc),
                  ctypes.byref(res), stream())
        e.record()
        torch.cuda.synchronize()
        if k >= 3:
            mtimes.append(s.elapsed_time(e))
    mms = float(np.median(mtimes))
    nr = float(torch.linalg.norm(xr))
    err64 = float(torch.linalg.norm(x64 - xr)) / nr
    errm = float(torch.linalg.norm(x - xr)) / nr
    del ctx
    return {"ms_per_solve": ms, "solves_per_s": 1000.0 / ms, "iterations": iters, "status": status,
            "elements": n * n, "nodes": (n + 1) ** 2, "algorithmic_bytes": byts,
            "achieved_gbs": byts / ms / 1e6, "frac_of_hbm": byts / ms / 1e6 / hbm, "rel_err_fp64": err64,
            "mixed": {"ms_per_solve": mms, "solves_per_s": 1000.0 / mms, "speedup_vs_fp64": ms / mms,
                      "cycles": cyc.value, "inner_iterations_per_cycle": 8, "fp64_relres": res.value,
                      "rel_err": errm}}


def poisson_sweep():
    """Poisson solve times on 2^k x 2^k Q1 meshes, k = 4..12 (16 .. 16.8M
    elements, the reference README's sweep sizes)."""
    return {f"poisson_{2 ** k}x{2 ** k}_q1": poisson(2 ** k) for k in range(4, 13)}


def serving(count, steps, plain_sample=128):
    """Request stream of independent wall-bounded solves (sizes uniform over
    32^2..256^2 Q1, viscosity log-uniform 1e-3..1e-1, Fourier initial velocity,
    `steps` steps each): the plain FP64 path (one request at a time on the
    whole device; timed on the first `plain_sample` requests, whose sizes
    follow the same distribution) against the continuous-batching server in
    FP64, saturated (all requests at t = 0) and under Poisson arrivals at
    50 %, 70 % and 90 % of the saturated throughput, and the server in mixed
    precision (mixed pressure solve), saturated. Latency = completion -
    arrival (plain: service time)."""
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")  # streams on separate hardware queues
    from jax_fem_cfd_b200.serving import Server, make_requests, run_plain
    reqs = make_requests(count, seed=0, steps=steps)
    srv = Server(keep_results=False)
    srv.prewarm(reqs)
    bad = lambda d: sum(1 for x in d if x["status"] != 0)
    sample = reqs[:min(plain_sample, count)]
    dp, plain = run_plain(sample, srv)
    ds, fixed = srv.run(reqs, realtime=False)
    tune = srv.autotune(reqs)
    srv.prewarm(reqs)
    ds2, sat = srv.run(reqs, realtime=False)
    out = {"workload": f"{count} requests x {steps} steps, Q1 {{32,64,128,256}}^2 wall-bounded",
           "plain": dict(plain, failed=bad(dp), sample=f"first {len(sample)} requests of the stream"),
           "served_saturated_untuned": dict(fixed, failed=bad(ds)),
           "autotune": tune, "served_saturated": dict(sat, failed=bad(ds2)),
           "speedup_solves_per_s": sat["solves_per_s"] / plain["solves_per_s"]}
    for frac in (0.5, 0.7, 0.9):
        rate = frac * sat["solves_per_s"]
        dr, m = srv.run(make_requests(count, seed=0, steps=steps, rate=rate))
        out[f"served_poisson_{int(frac * 100)}pct"] = dict(m, arrival_rate_per_s=rate, failed=bad(dr))
    del srv
    import torch
    torch.cuda.empty_cache()
    # packed launches: every size's requests as members of one persistent kernel per chunk
    from jax_fem_cfd_b200.serving import PackedServer
    ps = PackedServer(share=tune["picked"], keep_results=False)
    ptune = ps.autotune(reqs)
    out["autotune_packed"] = ptune
    plan = ps.prewarm(reqs)
    ps.run(reqs[:min(16, count)], realtime=False)  # first launches of each pack
    dpk, pk = ps.run(reqs, realtime=False)
    out["served_saturated_packed"] = dict(pk, failed=bad(dpk), members_per_size=plan)
    out["speedup_packed_solves_per_s"] = pk["solves_per_s"] / plain["solves_per_s"]
    for frac in (0.5, 0.9):
        rate = frac * pk["solves_per_s"]
        dr, m = ps.run(make_requests(count, seed=0, steps=steps, rate=rate))
        out[f"served_packed_poisson_{int(frac * 100)}pct"] = dict(m, arrival_rate_per_s=rate, failed=bad(dr))
    for p in ps.packs.values():
        p.close()
    del ps
    torch.cuda.empty_cache()
    mx = Server(keep_results=False, precision="mixed", share=tune["picked"])
    mx.prewarm(reqs)
    mx.run(reqs[:min(16, count)], realtime=False)  # graph builds of the mixed solves, once per pooled solver
    dm, msat = mx.run(reqs, realtime=False)
    out["served_saturated_mixed"] = dict(msat, failed=bad(dm))
    out["speedup_mixed_solves_per_s"] = msat["solves_per_s"] / plain["solves_per_s"]
    return out


def inverse(reps=3, adam_iters=5):
    """Differentiable inverse transport (128^2 Q1 unit square, all walls,
    nu 1e-3, scalar diffusivity 1e-4 with SUPG, dt 0.01, 150 steps, learnable
    FP32 initial velocity, adjoint gradient with a checkpoint every 10 steps):
    device time of the loss alone and of loss + gradient (CUDA events on the
    launching stream; the working set is L2-resident, so no flush), the
    gradient against a central difference along a seeded direction, and the
    loss over a few Adam iterations."""
    import torch

    from jax_fem_cfd_b200.solvers.inverse_transport import InverseTransport
    prob = InverseTransport()
    u0 = prob.initial_velocity()
    prob.value_and_grad(u0)

    def timed(fn):
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms))

    with torch.no_grad():
        fwd_ms = timed(lambda: prob.loss(u0))
    grad_ms = timed(lambda: prob.value_and_grad(u0))
    u64 = u0.to(torch.float64)
    L, g = prob.value_and_grad(u64)
    d = torch.randn(u64.numel(), generator=torch.Generator().manual_seed(7), dtype=torch.float64).to(u64.device)
    eps = 3e-4
    with torch.no_grad():
        fd = (float(prob.loss(u64 + eps * d)) - float(prob.loss(u64 - eps * d))) / (2 * eps)
    vjp = float((g * d).sum())
    p = u0.clone().requires_grad_(True)
    opt = torch.optim.Adam([p], lr=0.01)
    hist = []
    for _ in range(adam_iters):
        opt.zero_grad()
        Lk = prob.loss(p)
        Lk.backward()
        opt.step()
        hist.append(float(Lk.detach()))
    with torch.no_grad():
        hist.append(float(prob.loss(p)))
    return {"inverse_transport_128x128_q1": {
        "workload": "128^2 Q1 unit square, all walls, nu 1e-3, D 1e-4 (SUPG), dt 0.01, 150 steps, "
                    "checkpoint every 10 steps, FP32 initial velocity N(0, 0.1) seed 0, FP64 solves at tol 1e-10",
        "forward_ms": fwd_ms, "loss_and_gradient_ms": grad_ms, "gradients_per_s": 1e3 / grad_ms,
        "gradient_over_forward": grad_ms / fwd_ms,
        "fd_check": {"direction": "N(0,1) seed 7", "eps": eps, "adjoint": vjp, "central_difference": fd,
                     "rel_err": abs(vjp - fd) / abs(fd)},
        "adam_lr_0.01_loss": hist}}


def cavity_config_64(mod):
    """64^2 Q1 lid-driven cavity on the unit square, all walls Dirichlet, MG-PCG
    (final mesh 4 x 4) at tol 1e-8, pinned pressure."""
    return mod.Config(mesh="simple", solver="standard",
                      mesh_config=mod.SimpleMeshConfig(num_elem=[64, 64], domain_size=[1.0, 1.0], shape_func_ord=1,
                                                       periodic=False),
                      solver_config=mod.StandardSolverConfig(dirichlet_faces=[0, 1, 2, 3], symmetry_faces=[],
                                                             outlet_faces=[], streamline_diff=False, solver_tol=1e-8,
                                                             set_zeroP=True, pressure_precond="multigrid",
                                                             final_multigrid_mesh=[4, 4]))


def cavity(steps=200, warmup=3, cpu_steps=40):
    """The lid-driven cavity: 64^2 Q1, Re 100 (lid u = 1 including the corner
    nodes, mu = 0.01, rho = 1), dt 0.01, zero initial fields, 200 steps. Device
    time of the 200 steps with CUDA events (each step: the boundary integral
    and fem_step4), after `warmup` steps from which the fields are reset to
    zero; the numpy oracle, 1 thread, on the first `cpu_steps` steps beside it.
    The working set is L2-resident (no flush): this is the latency-bound end of
    the path."""
    import torch
    from threadpoolctl import threadpool_limits

    import oracle.simulation as osim
    from jax_fem_cfd_b200.setup import simulation as sim

    def prepare(mod):
        compute, timestep, nc, sn, h, nn, gd, Ud = mod.setup(cavity_config_64(mod))
        Ud = mod.set_face_velocity(Ud, sn[2], gd, 1.0, nn, var=1)
        return compute, timestep, nn, Ud

    compute, timestep, nn, Ud = prepare(sim)
    solver = timestep.solver
    bufs = [(torch.zeros(2 * nn, dtype=torch.float64, device="cuda"),
             torch.zeros(nn, dtype=torch.float64, device="cuda")) for _ in range(2)]
    its = []

    def run(k):
        for s in range(k):
            (U, P), o = bufs[s % 2], bufs[(s + 1) % 2]
            Fp, F = compute(Ud, None, s * 0.01, (s + 1) * 0.01)
            _, _, ui, pi = solver.step(U, P, 0.01, 1.0, 0.01, Ud, Fp, F, out=o)
            its.append((ui, pi))

    run(warmup)
    for U, P in bufs:
        U.zero_()
        P.zero_()
    its.clear()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run(steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    it = np.array([(int(a), int(b)) for a, b in its])
    with threadpool_limits(1):
        ocompute, otimestep, onn, oUd = prepare(osim)
        U, P = np.zeros(2 * onn), np.zeros(onn)
        t0 = time.perf_counter()
        for s in range(cpu_steps):
            Fp, F = ocompute(oUd, None, s * 0.01, (s + 1) * 0.01)
            U, P, _, _ = otimestep(U, P, 0.01, 1.0, 0.01, oUd, Fp, F)
        cpu_el = time.perf_counter() - t0
    return {"cavity_64x64_q1_re100": {
        "workload": "64^2 Q1 lid-driven cavity, Re 100 (corners on the lid), dt 0.01, 200 steps from zero, FP64, "
                    "MG-PCG tol 1e-8", "steps_per_s": steps / (ms * 1e-3), "ms_per_step": ms / steps,
        "status": int(solver.status.max()), "momentum_iters_mean": float(it[:, 0].mean()),
        "pressure_iters_mean": float(it[:, 1].mean()),
        "cpu_baseline": {"value": cpu_steps / cpu_el, "unit": "steps/s", "cores": 1, "kind": "port",
                         "sample": f"first {cpu_steps} steps of the same workload, numpy oracle, 1 thread"}}}


def mg3_vcycle(nx=256, reps=20, warmup=3):
    """The hex8 multigrid V-cycle of config 3's pressure solve, alone: the
    channel's pinned-pressure hierarchy (nx x nx/4 x nx/4 elements, 4 levels,
    Chebyshev degree 3), FP64, launched directly (fem_mg_vcycle; inside the
    PCG the same kernels run from a CUDA graph with a device-side loop, which
    profilers cannot split into kernels). A seeded rhs; device time per
    V-cycle with CUDA events, an L2-sized buffer written between cycles. The
    Chebyshev step kernel k_mg3_step on the finest level moves 48 algorithmic
    bytes per node (x_in, r, d, 1/D read; d, x_out written)."""
    import torch

    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr, stream
    from jax_fem_cfd_b200.setup import simulation as sim
    cfg = sim.Config(mesh="simple", solver="standard",
                     mesh_config=sim.SimpleMeshConfig(num_elem=[nx, nx // 4, nx // 4], domain_size=[4.0, 1.0, 1.0],
                                                      shape_func_ord=1, periodic=False),
                     solver_config=sim.StandardSolverConfig(dirichlet_faces=[0, 2, 3, 4, 5], symmetry_faces=[],
                                                            outlet_faces=[1], streamline_diff=False, solver_tol=1e-8,
                                                            set_zeroP=True, pressure_precond="multigrid",
                                                            final_multigrid_mesh=[nx // 8, nx // 32, nx // 32]))
    compute, timestep, nc, sn, h, nn, gd, Ud = sim.setup(cfg)
    ctx = timestep.solver.ctx
    r = torch.as_tensor(np.random.default_rng(0).standard_normal(nn), device="cuda")
    z = torch.empty_like(r)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    for _ in range(warmup):
        _lib.call("fem_mg_vcycle", ctx.handle, ptr(r), ptr(z), stream())
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.call("fem_mg_vcycle", ctx.handle, ptr(r), ptr(z), stream())
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return {"workload": f"hex8 channel {nx}x{nx // 4}x{nx // 4} pressure V-cycle (4 levels, Chebyshev degree 3, FP64)",
            "nodes": nn, "ms_per_vcycle_median": float(np.median(ms)), "reps": reps,
            "finest_step_algorithmic_bytes": 48 * nn, "finite": bool(torch.isfinite(z).all())}


def cg_trace(size=256):
    """Phase timeline of one pressure solve of the Taylor-Green step (size^2
    Q2, after 5 warm-up steps): CTA 0 of the persistent solvers stamps
    %globaltimer at every grid (tag 31) or team (tag 30) barrier and at the
    multigrid phase marks (fem_ctx_set_trace), and the gaps between
    consecutive marks are summed by (from, to) tag pair. The trace costs a few
    percent of the solve; the totals are for reading the phase structure, not
    a bench value."""
    import collections

    import torch

    import jax_fem_cfd_b200.setup.simulation as sim
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr
    compute, timestep, nc, sn, h, nn, gd, Ud = sim.setup(tg_config(sim, size))
    U0, P0 = tg_initial(nc.cpu().numpy())
    U, P = torch.as_tensor(U0).cuda(), torch.as_tensor(P0).cuda()
    Fp, F = compute(Ud, None, 0.0, 1e-3)
    for _ in range(5):
        U, P, ui, pi = timestep(U, P, 1e-3, 1.0, 0.01, Ud, Fp, F)
    torch.cuda.synchronize()
    ctx = timestep.solver.ctx
    cap = 1 << 16
    buf = torch.zeros(cap, dtype=torch.int64, device="cuda")
    _lib.call("fem_ctx_set_trace", ctx.handle, ptr(buf), cap)
    U, P, ui, pi = timestep(U, P, 1e-3, 1.0, 0.01, Ud, Fp, F)
    torch.cuda.synchronize()
    _lib.call("fem_ctx_set_trace", ctx.handle, None, 0)
    b = buf.cpu().numpy().astype(np.uint64)
    v = b[1:int(b[0]) + 1]
    tag = (v >> np.uint64(56)).astype(int)
    t = (v & np.uint64((1 << 56) - 1)).astype(np.int64)
    pairs = collections.defaultdict(list)
    for k in range(len(t) - 1):
        pairs[(int(tag[k]), int(tag[k + 1]))].append((t[k + 1] - t[k]) / 1e3)
    rows = sorted(pairs.items(), key=lambda kv: -sum(kv[1]))
    return {"workload": f"Taylor-Green {size}x{size} Q2, one step's BiCGSTAB and MG-PCG launches",
            "iterations": {"momentum": int(ui), "pressure": int(pi)}, "marks": int(len(t)),
            "span_us": float((t[-1] - t[0]) / 1e3),
            "pairs": [{"from": a, "to": b_, "count": len(x), "mean_us": float(np.mean(x)), "total_us": float(np.sum(x))}
                      for (a, b_), x in rows]}


def channel3d(steps=100, warmup=3, preconds=("jacobi", "approx_inv", "multigrid", "multigrid_mixed"), nx=256):
    """3D channel: hex8 256 x 64 x 64 on [0,4] x [0,1] x [0,1] (1,048,576
    elements, 1,090,625 nodes), parabolic inflow u = 16 y(1-y) z(1-z) on x = 0,
    zero-traction outlet (P = 0) on x = 4, no-slip walls, Re 200 (mu = 1/200,
    rho = 1), dt 2e-3, zero initial fields, tol 1e-8. Pressure solves: Jacobi
    and approx_inv PCG (FP64, the preconditioners the reference's 3D path
    accepts), the hex8 multigrid PCG (4 levels down to 32 x 8 x 8 elements,
    Chebyshev degree 3; FP64), and the same multigrid as FP32 inner iterations
    inside FP64 refinement to 1e-8 ("multigrid_mixed", the configuration the
    workload names). One step = the boundary integral plus fem_step4; device
    time with CUDA events, working set beyond L2 (the Gauss factors of the
    convection alone are 268 MB). Each arm's final U and P are compared with
    the first arm's (FP64, same tolerance). nx < 256 runs the same channel on
    nx x nx/4 x nx/4 elements (the multigrid still has 4 levels), for
    profiling on a smaller case."""
    import torch

    from jax_fem_cfd_b200.setup import simulation as sim
    out = {}
    ref = None
    for pc in preconds:
        prec, extra = pc, {}
        if pc.startswith("multigrid"):
            prec = "multigrid"
            extra = {"final_multigrid_mesh": [nx // 8, nx // 32, nx // 32]}
            if pc.endswith("mixed"):
                extra["precision"] = "mixed"
        cfg = sim.Config(mesh="simple", solver="standard",
                         mesh_config=sim.SimpleMeshConfig(num_elem=[nx, nx // 4, nx // 4], domain_size=[4.0, 1.0, 1.0],
                                                          shape_func_ord=1, periodic=False),
                         solver_config=sim.StandardSolverConfig(dirichlet_faces=[0, 2, 3, 4, 5], symmetry_faces=[],
                                                                outlet_faces=[1], streamline_diff=False,
                                                                solver_tol=1e-8, set_zeroP=True, pressure_precond=prec,
                                                                **extra))
        compute, timestep, nc, sn, h, nn, gd, Ud = sim.setup(cfg)
        y, z = nc[sn[3], 1], nc[sn[3], 2]
        Ud = sim.set_face_velocity(Ud, sn[3], gd, 16 * y * (1 - y) * z * (1 - z), nn, var=1)
        solver = timestep.solver
        dt, mu = 2e-3, 1.0 / 200
        bufs = [(torch.zeros(3 * nn, dtype=torch.float64, device="cuda"),
                 torch.zeros(nn, dtype=torch.float64, device="cuda")) for _ in range(2)]
        its = []

        def run(k, t0):
            for s in range(k):
                (U, P), o = bufs[(t0 + s) % 2], bufs[(t0 + s + 1) % 2]
                Fp, F = compute(Ud, None, (t0 + s) * dt, (t0 + s + 1) * dt)
                _, _, ui, pi = solver.step(U, P, dt, 1.0, mu, Ud, Fp, F, out=o)
                its.append((ui, pi))

        run(warmup, 0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run(steps, warmup)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        it = np.array([(int(a), int(b)) for a, b in its[warmup:]])
        st = int(solver.status.max())
        U, P = bufs[(warmup + steps) % 2]
        out[pc] = {"steps_per_s": steps / (ms * 1e-3), "ms_per_step": ms / steps, "status": st,
                   "momentum_iters_mean": float(it[:, 0].mean()), "pressure_iters_mean": float(it[:, 1].mean()),
                   "pressure_iters_first_last": [int(it[0, 1]), int(it[-1, 1])],
                   "u_max_after": float(U[:nn].max()), "finite": bool(torch.isfinite(U).all())}
        if pc.endswith("mixed"):
            out[pc]["pressure_iters_are"] = f"FP64 refinement cycles ({_mixed_inner()} FP32 multigrid-PCG iterations each)"
        if ref is None:
            ref = (U.clone(), P.clone())
        else:
            out[pc]["rel_err_vs_" + preconds[0]] = {
                "U": float(torch.linalg.vector_norm(U - ref[0]) / torch.linalg.vector_norm(ref[0])),
                "P": float(torch.linalg.vector_norm(P - ref[1]) / torch.linalg.vector_norm(ref[1]))}
        del compute, timestep, solver, bufs, nc, sn, gd, Ud
        torch.cuda.empty_cache()
    del ref
    return {f"channel3d_hex8_{nx}x{nx // 4}x{nx // 4}": {
        "workload": "hex8 256x64x64 channel, parabolic inflow, outlet, Re 200, dt 2e-3, tol 1e-8, zero start",
        "timed_steps": steps, "warmup": warmup, **out}}


def poisson_and_matvec(args):
    """Reference-published GPU figures on their own sizes (README.md:28-41):
    MG-PCG Poisson solve on 1024x1024 Q1 elements and the EBE matvec on
    4096x4096 Q1 elements (beyond L2: a true HBM-roofline kernel)."""
    r = poisson(1024)
    out = {"poisson_1024x1024_q1": dict(metric="Poisson solves/s (MG-PCG, tol 1e-8)", value=r["solves_per_s"],
                                        reference_published_ms_unnamed_gpu=28.0, **r)}
    out.update(matvec())
    return out


def matvec():
    """EBE Laplacian matvec, 4096x4096 Q1 (16.8M elements, 134 MB per vector)."""
    import torch

    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import Context, Mesh, ptr, stream
    out = {}
    hbm, _ = measured_peaks()
    rng = np.random.default_rng(0)
    n = 4096
    ctx = Context(Mesh(0, False, n, n, 1, 1.0, 1.0))
    Le = ctx.element_data()[4].reshape(-1).contiguous()
    xv = torch.as_tensor(rng.standard_normal(ctx.nn), device="cuda")
    yv = torch.empty_like(xv)
    for _ in range(3):
        _lib.call("fem_ebe_apply", ctx.handle, 1, ptr(xv), ptr(yv), 1.0, ptr(Le), 0.0, None, 0, 0.0, None, stream())
    # 20 back-to-back applies per event pair (x and y, 268 MB, exceed L2), so the
    # host call is off the critical path; each apply includes its table build
    times, reps = [], 20
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            _lib.call("fem_ebe_apply", ctx.handle, 1, ptr(xv), ptr(yv), 1.0, ptr(Le), 0.0, None, 0, 0.0, None,
                      stream())
        e.record()
        torch.cuda.synchronize()
        times.append(s.elapsed_time(e) / reps)
    ms = float(np.median(times))
    byts = 2 * ctx.nn * 8
    out["ebe_matvec_4096x4096_q1"] = {"ms_per_apply": ms, "elements": n * n, "algorithmic_bytes": byts,
                                      "achieved_gbs": byts / ms / 1e6, "frac_of_hbm": byts / ms / 1e6 / hbm,
                                      "reference_published_ms_unnamed_gpu": 4.5}
    del ctx
    return out


def cpu_baseline(n, steps):
    """The oracle (numpy FP64 restatement, 1 thread) on the same workload."""
    from threadpoolctl import threadpool_limits

    import oracle.simulation as osim
    with threadpool_limits(1):
        compute, timestep, nc, sn, h, nn, gd, Ud = osim.setup(tg_config(osim, n))
        U, P = tg_initial(nc)
        Fp, F = compute(Ud, None, 0, 0)
        t0 = time.perf_counter()
        for _ in range(steps):
            U, P, _, _ = timestep(U, P, 1e-3, 1.0, 0.01, Ud, Fp, F)
        el = time.perf_counter() - t0
    return {"value": steps / el, "unit": "steps/s", "cores": 1, "kind": "port",
            "sample": f"{steps} full NS steps of the same 256x256 Q2 workload, numpy oracle, 1 thread"}


def run_reference(args):
    """--impl reference: the oracle port of the reference's CPU path, all host
    threads, same workload and metric."""
    import oracle.simulation as osim
    n = args.size
    compute, timestep, nc, sn, h, nn, gd, Ud = osim.setup(tg_config(osim, n))
    U, P = tg_initial(nc)
    Fp, F = compute(Ud, None, 0, 0)
    for _ in range(min(args.warmup, 1)):
        U, P, _, _ = timestep(U, P, 1e-3, 1.0, 0.01, Ud, Fp, F)
    # bounded sample: at most REFERENCE_SAMPLE_S seconds of steps (a rate, so any
    # number of whole steps measures it), at least one step
    t0 = time.perf_counter()
    done = 0
    while done < args.steps:
        U, P, _, _ = timestep(U, P, 1e-3, 1.0, 0.01, Ud, Fp, F)
        done += 1
        if time.perf_counter() - t0 > REFERENCE_SAMPLE_S:
            break
    el = time.perf_counter() - t0
    v = done / el
    line = {"metric": "NS steps/s", "value": v, "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * el / done, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic TG initial field)",
            "impl": "reference",
            "config": {k: v_ for k, v_ in WORKLOAD.items() if k not in ("nex", "ney")} | {"parallelism": "none (CPU)"},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"{done} full NS steps of the workload (bounded at {REFERENCE_SAMPLE_S:.0f} s), "
                                       "numpy oracle, all host threads"},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--no-extra", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--only", choices=["matvec", "poisson", "poisson_sweep", "serving", "inverse", "channel3d",
                                       "cavity", "tg_mixed", "mg3_vcycle", "cg_trace"],
                    help="run one secondary measurement alone and print it (poisson: the --size mesh)")
    ap.add_argument("--requests", type=int, default=1024, help="--only serving: requests in the stream")
    ap.add_argument("--channel-nx", type=int, default=256, help="--only channel3d: elements along x (y, z: nx / 4)")
    ap.add_argument("--preconds", default="jacobi,approx_inv,multigrid,multigrid_mixed",
                    help="--only channel3d: pressure solves to run")
    ap.add_argument("--request-steps", type=int, default=200, help="--only serving: steps per request")
    args = ap.parse_args()
    if args.only:
        fn = {"matvec": matvec, "poisson_sweep": poisson_sweep,
              "poisson": lambda: {f"poisson_{args.size}x{args.size}_q1": poisson(args.size)},
              "serving": lambda: serving(args.requests, args.request_steps), "inverse": inverse,
              "channel3d": lambda: channel3d(args.steps, preconds=tuple(args.preconds.split(",")),
                                             nx=args.channel_nx), "cavity": cavity,
              "tg_mixed": lambda: tg_mixed_long(500, args.size),
              "mg3_vcycle": lambda: mg3_vcycle(args.channel_nx), "cg_trace": lambda: cg_trace(args.size)}[args.only]
        print(json.dumps(fn()))
        return
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    r = run_ours(args, rank, world, local_rank)
    extra = {}
    if not args.no_extra and rank == 0:
        extra = poisson_and_matvec(args)
    mixed = None
    if not args.no_extra and rank == 0 and world == 1:
        mixed = tg_mixed(args, r["final"], r["coords"])
    del r["final"]
    hbm, src = measured_peaks()
    K = args.steps
    ms_step = r["total_ms"] / K
    value = whole_job_rate(world, K, r["total_ms"])
    stage = dict(zip(STAGES, r["stage_ms"]))
    stage_tot = sum(r["stage_ms"])
    share = {k: v / stage_tot for k, v in stage.items()} if stage_tot > 0 else {}
    p_iters = [pi for _, pi in r["iters"]]
    u_iters = [ui for ui, _ in r["iters"]]
    cg_bytes = np.mean([cg_algorithmic_bytes(r["level_nn"], it, None) for it in p_iters])
    cg_ms = stage["pressure_pcg"]
    traffic = None
    tp = os.path.join(ROOT, "profiles", "k_cg_tg256_traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get("dram_bytes_per_launch")
        except Exception:
            traffic = None
    ctx = r["ctx"]
    bi_bytes = np.mean([bicgstab_algorithmic_bytes(ctx.nn, ctx.ne, ctx.nen, 2, it) for it in u_iters])
    line = {
        "metric": "NS steps/s", "value": value, "unit": "steps/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic Taylor-Green initial field)",
        "config": {**{k: v for k, v in WORKLOAD.items() if k not in ("nex", "ney")},
                   "unique_nodes": r["nn"], "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "flushed between timed steps (256 MiB write)"},
        "e2e": {"value": whole_job_rate(world, K, r["e2e_ms"]), "unit": "steps/s", "h2d_bytes_per_step": r["h2d"],
                "d2h_bytes_per_step": r["d2h"]},
        "gpu_launches": int(r["launches"]),
        "roofline": {"kernel": "k_cg<1,0> (persistent MG-PCG pressure solve, Q2, mean-zero)", "bound": "hbm",
                     "achieved": cg_bytes / (cg_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                     "frac": cg_bytes / (cg_ms * 1e-3) / 1e9 / hbm, "traffic": traffic,
                     "algorithmic_bytes_per_launch": cg_bytes, "avg_launch_ms": cg_ms,
                     "peak_source": src},
        "roofline_momentum": {"kernel": "k_bicgstab<1,2> (Q2, 2 velocity components)", "achieved": bi_bytes / (stage["momentum_bicgstab"] * 1e-3) / 1e9,
                              "peak": hbm, "unit": "GB/s",
                              "frac": bi_bytes / (stage["momentum_bicgstab"] * 1e-3) / 1e9 / hbm},
        "stage_ms": stage, "stage_share": share,
        "iterations": {"momentum_mean": float(np.mean(u_iters)), "pressure_mean": float(np.mean(p_iters))},
        "clocks": r["clocks"],
        **extra,
    }
    if mixed is not None:
        line["mixed"] = dict(mixed, speedup_vs_fp64=mixed["steps_per_s"] / value)
    if rank == 0 and world == 1 and args.cpu_steps > 0:
        line["cpu_baseline"] = cpu_baseline(args.size, args.cpu_steps)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
