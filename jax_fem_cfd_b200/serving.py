"""Serving: continuous batching of independent 2D wall-bounded flow solves.

A request is one Navier-Stokes problem on the unit square (Q1, all walls
no-slip, pressure pinned at node 0, MG-PCG pressure and BiCGSTAB momentum at
tol 1e-8), with its own mesh size, viscosity and divergence-free initial
velocity, run for a fixed number of 4-step projection steps (the step of
solvers/standard.py:148-165).

The request loop (`Server.run`) is continuous batching, not a queue:

- Requests arrive over time (Poisson arrivals, or all at t = 0). A request is
  admitted as soon as the device has room for it: a share of the cooperative
  CTA capacity (its solver kernels are persistent cooperative grids, and the
  grids of all admitted requests must fit on the device at once) and, when no
  pooled solver of its size is idle, the HBM a new one needs (free device
  memory against the footprint measured when the first solver of that size
  was built).
- Solvers (context, element matrices, multigrid hierarchy, boundary sets, the
  velocity / pressure ping-pong buffers) are pooled per mesh size and stay
  resident: a finished request hands its solver to the next request of that
  size, so nothing is allocated or freed while requests run.
- Every admitted request runs on its own CUDA stream, in chunks of steps; up to
  two chunks per request are queued at a time, so the requests' kernels
  overlap on the device and a new arrival is never behind a long queue. A
  chunk is one launch of a CUDA graph captured for the request at admission
  (fem_step4_graph: the chunk's steps with the request's dt and viscosity).
- The CTA cap of a request can be picked by `Server.autotune`, which serves a
  short sample of the stream under a few caps and keeps the fastest.
- precision="mixed" serves every request with the mixed-precision pressure
  solve (FP64 refinement around FP32 multigrid-PCG, one CUDA graph with a
  device-side loop per solve); its steps are launched directly (a step that
  launches its own graph is not captured into a chunk graph).
- A request's CTA share depends only on its mesh size, so its results are the
  same (bit for bit) alone and in any mix: the solver's reductions are
  deterministic for a given grid.

No reference counterpart: the reference runs one problem per process.
"""
import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .context import ptr

SIZES = (32, 64, 128, 256)


@dataclass
class Request:
    rid: int
    n: int                   # Q1 elements per side of the unit square
    nu: float                # kinematic viscosity (rho = 1, so mu = nu)
    steps: int
    dt: float
    arrival: float           # seconds after the start of the stream
    U0: np.ndarray = field(repr=False)  # (2 (n+1)^2,) initial velocity, component-major


def fourier_velocity(n, seed, kmax=8):
    """Divergence-free velocity on the (n+1)^2 nodes of the unit square: the
    curl of a stream function made of the Fourier modes 1 <= |k| <= kmax with
    seeded N(0,1) cosine and sine coefficients of amplitude 1/|k|^2, scaled to
    max |u| = 1. Returned as [u; v] (component-major, like the solver's U)."""
    rng = np.random.default_rng(seed)
    x = np.linspace(0.0, 1.0, n + 1)
    X, Y = np.meshgrid(x, x)  # node (i, j) -> row j, column i: node id j (n+1) + i
    u = np.zeros_like(X)
    v = np.zeros_like(X)
    for kx in range(-kmax, kmax + 1):
        for ky in range(0, kmax + 1):
            k2 = kx * kx + ky * ky
            if k2 == 0 or k2 > kmax * kmax or (ky == 0 and kx < 0):
                continue
            a, b = rng.standard_normal(2) / k2
            ph = 2.0 * np.pi * (kx * X + ky * Y)
            # psi = a cos(ph) + b sin(ph); u = dpsi/dy, v = -dpsi/dx
            d = 2.0 * np.pi * (-a * np.sin(ph) + b * np.cos(ph))
            u += d * ky
            v -= d * kx
    s = np.sqrt(u * u + v * v).max()
    s = s if s > 0 else 1.0
    return np.concatenate([u.ravel(), v.ravel()]) / s


def make_requests(count, seed=0, sizes=SIZES, nu_range=(1e-3, 1e-1), steps=200, rate=None, kmax=8, cfl=0.25):
    """Seeded request stream: size uniform over `sizes`, viscosity log-uniform
    over `nu_range`, Fourier initial velocity (seed = request id + seed), time
    step dt = cfl * h (|u| <= 1), arrivals Poisson at `rate` per second (all at
    t = 0 when rate is None)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        n = int(sizes[rng.integers(len(sizes))])
        nu = float(math.exp(rng.uniform(math.log(nu_range[0]), math.log(nu_range[1]))))
        if rate:
            t += float(rng.exponential(1.0 / rate))
        out.append(Request(i, n, nu, steps, cfl / n, t if rate else 0.0, fourier_velocity(n, seed + i, kmax)))
    return out


def cavity_config(n, precision="fp64"):
    """Wall-bounded unit square, Q1, all four faces Dirichlet (U_d = 0),
    pinned pressure, MG-PCG (final mesh 4 x 4) at tol 1e-8; precision "mixed"
    solves the pressure by FP64 refinement around FP32 multigrid-PCG."""
    from .setup import simulation as sim
    return sim.Config(mesh="simple", solver="standard",
                      mesh_config=sim.SimpleMeshConfig(num_elem=[n, n], domain_size=[1.0, 1.0], shape_func_ord=1,
                                                       periodic=False),
                      solver_config=sim.StandardSolverConfig(dirichlet_faces=[0, 1, 2, 3], symmetry_faces=[],
                                                             outlet_faces=[], streamline_diff=False, solver_tol=1e-8,
                                                             set_zeroP=True, pressure_precond="multigrid",
                                                             final_multigrid_mesh=[4, 4], precision=precision))


class Slot:
    """Pooled device state of one mesh size: the solver and its buffers."""

    def __init__(self, n, precision="fp64"):
        from .setup import simulation as sim
        _, timestep, *_rest = sim.setup(cavity_config(n, precision))
        U_d = _rest[-1]
        self.n = n
        self.solver = timestep.solver
        s = self.solver
        self.ud = s.u_full(U_d)
        nn = s.nn
        dev = s.ctx.dev
        self.U = [torch.zeros(2 * nn, dtype=torch.float64, device=dev) for _ in range(2)]
        self.P = [torch.zeros(nn, dtype=torch.float64, device=dev) for _ in range(2)]
        self.iters = torch.zeros(2, dtype=torch.int32, device=dev)
        self.U_host = torch.empty(2 * nn, dtype=torch.float64).pin_memory()
        self.P_host = torch.empty(nn, dtype=torch.float64).pin_memory()
        self.U0_host = torch.empty(2 * nn, dtype=torch.float64).pin_memory()
        self.status_host = torch.empty(2, dtype=torch.int32).pin_memory()
        if precision == "mixed":
            # the mixed pressure solve builds its FP32 hierarchy and its graph on
            # first use (with a device synchronisation): do it here, not while serving
            self.steps(0, 1, 1e-3, 1e-2, torch.cuda.current_stream())
            torch.cuda.synchronize()
            for b in self.U + self.P:
                b.zero_()

    def set_ctas(self, ctas):
        cap = ctypes.c_int(0)
        _lib.call("fem_ctx_set_max_ctas", self.solver.ctx.handle, int(ctas), ctypes.byref(cap))
        return cap.value

    def graph(self, steps, dt, mu):
        """A captured chunk of `steps` (even) steps from and back to buffer 0."""
        s = self.solver
        h = ctypes.c_void_p()
        _lib.call("fem_step4_graph", s.ctx.handle, ptr(self.U[0]), ptr(self.P[0]), ptr(self.U[1]), ptr(self.P[1]),
                  float(dt), 1.0, float(mu), ptr(self.ud), None, None, float(s.cfg.solver_tol), s.precond,
                  int(steps), ptr(self.iters), ptr(s.status), ctypes.byref(h))
        return h

    def steps(self, cur, k, dt, mu, stream):
        """k steps from buffer `cur`; returns the buffer holding the result."""
        s, h = self.solver, ctypes.c_void_p(stream.cuda_stream)
        for _ in range(k):
            nxt = 1 - cur
            _lib.call("fem_step4", s.ctx.handle, ptr(self.U[cur]), ptr(self.P[cur]), float(dt), 1.0, float(mu),
                      ptr(self.ud), None, None, float(s.cfg.solver_tol), s.precond, ptr(self.U[nxt]),
                      ptr(self.P[nxt]), ptr(self.iters), ptr(s.status), h)
            cur = nxt
        return cur


class _Active:
    __slots__ = ("req", "slot", "stream", "cur", "enq", "events", "final", "admitted", "ctas", "graph")

    def __init__(self, req, slot, stream, ctas):
        self.req, self.slot, self.stream, self.ctas = req, slot, stream, ctas
        self.cur, self.enq, self.events, self.final, self.admitted = 0, 0, [], None, 0.0
        self.graph = None


def ctas_for(n, share):
    """CTA share of a request of mesh size n: about one node per thread (the
    solver's own sizing for a dedicated device), capped at `share`."""
    nn = (n + 1) ** 2
    return max(1, min(share, -(-nn // 512)))


class Server:
    """Continuous-batching request loop over pooled solvers (see module doc).

    share: CTA cap of one request (the device capacity is SMs x resident
    solver CTAs per SM, 148 on a B200); chunk: steps per queued chunk;
    hbm_reserve: bytes kept free when building a new solver."""

    def __init__(self, share=37, chunk=10, hbm_reserve=2 << 30, keep_results=True, graphs=True, precision="fp64"):
        self.share, self.chunk, self.hbm_reserve = share, chunk + (chunk & 1), hbm_reserve
        self.precision = precision
        self.keep_results = keep_results
        self.graphs = graphs
        self.graph_error = None
        self.share_by_size = {}  # n -> fixed CTA share of that size, overriding the cap
        self.pool = {}        # n -> idle Slots
        self.footprint = {}   # n -> device bytes of one Slot
        self.streams = []
        self.capacity = None

    def _new_slot(self, n):
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        slot = Slot(n, self.precision)
        torch.cuda.synchronize()
        used = free0 - torch.cuda.mem_get_info()[0]
        self.footprint[n] = max(self.footprint.get(n, 0), used, 1 << 20)
        cap = slot.set_ctas(0)
        self.capacity = cap if self.capacity is None else min(self.capacity, cap)
        return slot

    def ctas(self, n):
        return self.share_by_size.get(n) or ctas_for(n, self.share)

    def autotune(self, requests, caps=(8, 16, 37, 74), sample=16, sample_steps=20):
        """Pick the CTA cap of one request by serving a sample of the stream:
        the first `sample` requests, cut to `sample_steps` steps each, all at
        t = 0, once per cap in `caps`; the cap with the most solves per second
        is kept (self.share). A per-size optimum of steps per second per CTA
        would favour tiny shares and leave the largest requests to set the
        makespan, so the tuning runs the actual mix. Returns the table."""
        import dataclasses
        trial = [dataclasses.replace(r, steps=min(r.steps, sample_steps), arrival=0.0) for r in requests[:sample]]
        keep = self.keep_results
        self.keep_results = False
        self.share_by_size = {}
        table = {}
        for cap in caps:
            self.share = cap
            self.prewarm(trial)
            self.run(trial, realtime=False)  # first pass: graph and stream set-up
            _, m = self.run(trial, realtime=False)
            table[cap] = m["solves_per_s"]
        self.share = max(table, key=table.get)
        self.keep_results = keep
        return {"picked": self.share, "sample_solves_per_s": table, "sample": f"{len(trial)} x {sample_steps} steps"}

    def warm(self, sizes):
        """Build one pooled solver per size before the clock starts."""
        for n in sizes:
            if not self.pool.get(n):
                self.pool.setdefault(n, []).append(self._new_slot(n))

    def prewarm(self, requests):
        """Build, before the clock starts, as many solvers per size as can run
        at once under the CTA capacity (at most one per request of that size),
        so the loop never builds one (building synchronises the device)."""
        sizes = sorted({r.n for r in requests})
        self.warm(sizes)
        for n in sizes:
            want = min(sum(r.n == n for r in requests), max(1, self.capacity // self.ctas(n)))
            have = len(self.pool[n])
            for _ in range(want - have):
                self.pool[n].append(self._new_slot(n))

    def _take_slot(self, n):
        idle = self.pool.setdefault(n, [])
        if idle:
            return idle.pop()
        if n in self.footprint and torch.cuda.mem_get_info()[0] < self.footprint[n] + self.hbm_reserve:
            return None
        return self._new_slot(n)

    def run(self, requests, realtime=True):
        """Serve `requests` (sorted by arrival); returns per-request records and
        the stream's metrics. realtime=False admits every request at t = 0."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        if self.capacity is None:
            self.warm(sorted({r.n for r in reqs}))
        pending, active, done = [], [], []
        used = 0
        nxt = 0
        free_streams = list(self.streams)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        while nxt < len(reqs) or pending or active:
            now = time.perf_counter() - t0
            while nxt < len(reqs) and (not realtime or reqs[nxt].arrival <= now):
                pending.append(reqs[nxt])
                nxt += 1
            # admission: FIFO, while the head fits in CTAs and memory
            while pending:
                r = pending[0]
                c = self.ctas(r.n)
                if used + c > self.capacity:
                    break
                slot = self._take_slot(r.n)
                if slot is None:
                    break
                pending.pop(0)
                if not free_streams:
                    st = torch.cuda.Stream()
                    self.streams.append(st)
                    free_streams.append(st)
                a = _Active(r, slot, free_streams.pop(), c)
                a.admitted = time.perf_counter() - t0
                slot.set_ctas(c)
                slot.U0_host.copy_(torch.from_numpy(r.U0))
                with torch.cuda.stream(a.stream):
                    slot.U[0].copy_(slot.U0_host, non_blocking=True)
                    slot.P[0].zero_()
                if self.graphs and r.steps >= self.chunk:
                    try:
                        a.graph = slot.graph(self.chunk, r.dt, r.nu)
                    except _lib.FemError as e:  # capture unsupported here: launch the steps directly
                        self.graphs, self.graph_error = False, str(e)
                used += c
                active.append(a)
            # feed and retire
            for a in list(active):
                a.events = [e for e in a.events if not e.query()]
                if a.enq < a.req.steps and len(a.events) < 2:
                    k = min(self.chunk, a.req.steps - a.enq)
                    if a.graph is not None and k == self.chunk and a.cur == 0:
                        _lib.call("fem_graph_launch", a.graph, ctypes.c_void_p(a.stream.cuda_stream))
                    else:
                        a.cur = a.slot.steps(a.cur, k, a.req.dt, a.req.nu, a.stream)
                    a.enq += k
                    ev = torch.cuda.Event()
                    ev.record(a.stream)
                    a.events.append(ev)
                    if a.enq == a.req.steps:
                        s = a.slot
                        with torch.cuda.stream(a.stream):
                            s.U_host.copy_(s.U[a.cur], non_blocking=True)
                            s.P_host.copy_(s.P[a.cur], non_blocking=True)
                            s.status_host.copy_(s.solver.status, non_blocking=True)
                        a.final = torch.cuda.Event()
                        a.final.record(a.stream)
                elif a.final is not None and a.final.query():
                    t = time.perf_counter() - t0
                    s = a.slot
                    rec = {"rid": a.req.rid, "n": a.req.n, "arrival": a.req.arrival, "admitted": a.admitted,
                           "done": t, "latency": t - (a.req.arrival if realtime else 0.0), "ctas": a.ctas,
                           "status": int(s.status_host[0]) | int(s.status_host[1])}
                    if self.keep_results:
                        rec["U"] = s.U_host.numpy().copy()
                        rec["P"] = s.P_host.numpy().copy()
                    done.append(rec)
                    if a.graph is not None:
                        _lib.call("fem_graph_destroy", a.graph)
                    active.remove(a)
                    used -= a.ctas
                    self.pool[s.n].append(s)
                    free_streams.append(a.stream)
        wall = time.perf_counter() - t0
        lat = np.array([d["latency"] for d in done])
        steps = sum(r.steps for r in reqs)
        return done, {"requests": len(done), "wall_s": wall, "solves_per_s": len(done) / wall,
                      "steps_per_s": steps / wall, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                      "p99_ms": float(np.percentile(lat, 99) * 1e3), "capacity_ctas": self.capacity,
                      "share_ctas": {n: self.ctas(n) for n in sorted({r.n for r in reqs})},
                      "graphs": self.graphs, "graph_error": self.graph_error}


class Pack:
    """k pooled solvers of one mesh size advanced together (fem_pack_step):
    one persistent cooperative launch per call runs every active member's
    steps, each member on its own group of `ctas` CTAs with its own barriers,
    so a member's results are those of its solver run alone on `ctas` CTAs,
    bit for bit. Members join and leave between calls."""

    def __init__(self, n, k, ctas):
        self.n, self.k, self.ctas = n, k, ctas
        self.slots = [Slot(n) for _ in range(k)]
        for sl in self.slots:
            sl.set_ctas(ctas)
        s0 = self.slots[0].solver
        dev = s0.ctx.dev
        self.stat = torch.zeros(5 * k, dtype=torch.int32, device=dev)
        self.stat_host = torch.zeros(5 * k, dtype=torch.int32).pin_memory()
        vp = lambda xs: (ctypes.c_void_p * k)(*[ctypes.c_void_p(x) for x in xs])
        h = ctypes.c_void_p()
        _lib.call("fem_pack_create", vp([sl.solver.ctx.handle.value for sl in self.slots]), k,
                  vp([sl.U[0].data_ptr() for sl in self.slots]), vp([sl.P[0].data_ptr() for sl in self.slots]),
                  vp([sl.U[1].data_ptr() for sl in self.slots]), vp([sl.P[1].data_ptr() for sl in self.slots]),
                  vp([sl.ud.data_ptr() for sl in self.slots]), ptr(self.stat), float(s0.cfg.solver_tol),
                  int(s0.precond), ctypes.byref(h))
        self.handle = h

    def step(self, dt, mu, steps, cur, stream):
        """steps[m] steps of member m (0: idle) from buffer cur[m], one launch
        on `stream`; member m's result is then in buffer cur[m] ^ (steps[m] & 1)."""
        k = self.k
        _lib.call("fem_pack_step", self.handle, (ctypes.c_double * k)(*dt), (ctypes.c_double * k)(*mu),
                  (ctypes.c_int * k)(*steps), (ctypes.c_int * k)(*cur), ctypes.c_void_p(stream.cuda_stream))

    def close(self):
        if self.handle is not None:
            _lib.call("fem_pack_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Member:
    __slots__ = ("req", "cur", "left", "admitted", "final", "result")

    def __init__(self):
        self.req, self.cur, self.left, self.admitted, self.final, self.result = None, 0, 0, 0.0, None, None


class PackedServer:
    """Continuous batching with packed launches: the requests of one mesh size
    are members of that size's Pack, and each launch advances the pack's active
    members by one chunk of steps (one persistent kernel for the whole chunk,
    no per-step launches and no per-request graphs). Launches are elastic: a
    launch holds only its active members' CTAs, and every size's pack draws on
    one budget of co-resident CTAs (the device capacity), so when one size's
    requests run out, the others take its CTAs. A request is admitted into a
    free member of its size's pack between that pack's launches; the packs are
    served oldest work first. Results are each request's solo results on its
    CTA count, bit for bit, whatever the mix."""

    def __init__(self, share=16, chunk=10, keep_results=True, members=None, ctas_by_size=None):
        self.share, self.chunk, self.keep_results = share, chunk, keep_results
        self.members = dict(members or {})  # n -> members of that size's pack (overrides the default)
        self.ctas_by_size = dict(ctas_by_size or {})  # n -> CTAs per member (overrides the share)
        self.packs = {}
        self.capacity = None

    def ctas(self, n):
        return self.ctas_by_size.get(n) or ctas_for(n, self.share)

    def autotune(self, requests, candidates=None, sample=64):
        """Pick the CTAs per member of each size by serving a sample of the
        stream (its first `sample` requests at their full length, all at t = 0)
        under a few maps and keeping the one with the most solves per second
        (self.ctas_by_size). The default candidates range from the stream
        server's share down to one CTA for the smallest meshes: packed members
        run whole steps inside one launch, so fewer CTAs per member and more
        members can win where a launch per step could not. Returns the table."""
        cands = candidates or [{}, {32: 1, 64: 2, 128: 4, 256: 8}, {32: 1, 64: 1, 128: 2, 256: 4},
                               {32: 1, 64: 2, 128: 8, 256: 16}, {32: 2, 64: 4, 128: 8, 256: 8}]
        trial = requests[:sample]
        sizes = sorted({r.n for r in requests})
        keep = self.keep_results
        self.keep_results = False
        table = []
        for cb in cands:
            self.ctas_by_size = dict(cb)
            self.close()
            self.prewarm(trial)
            self.run(trial[:8], realtime=False)
            _, m = self.run(trial, realtime=False)
            table.append((m["solves_per_s"], cb))
        best = max(table, key=lambda t: t[0])[1]
        self.ctas_by_size = dict(best)
        self.close()
        self.keep_results = keep
        return {"picked": {n: self.ctas(n) for n in sizes},
                "sample_solves_per_s": [{"ctas": {n: cb.get(n) or ctas_for(n, self.share) for n in sizes},
                                         "solves_per_s": v} for v, cb in table],
                "sample": f"first {len(trial)} requests"}

    def close(self):
        for p in self.packs.values():
            p.close()
        self.packs = {}

    def plan(self, requests):
        """Members per size: as many as the requests of that size, up to what
        the CTA capacity can run at once (and 64, the most a pack takes)."""
        sizes = sorted({r.n for r in requests})
        probe = Slot(sizes[0])
        cap = ctypes.c_int(0)
        _lib.call("fem_ctx_set_max_ctas", probe.solver.ctx.handle, 0, ctypes.byref(cap))
        del probe
        self.capacity = cap.value  # the packed kernel holds one CTA per SM, like the solver kernels
        return {n: self.members.get(n) or max(1, min(sum(r.n == n for r in requests), 64,
                                                     self.capacity // self.ctas(n))) for n in sizes}

    def prewarm(self, requests):
        """Build the packs (solvers, hierarchies, pack objects) before the clock."""
        plan = self.plan(requests)
        for n, k in plan.items():
            p = self.packs.get(n)
            if p is None or p.k != k or p.ctas != self.ctas(n):
                if p is not None:
                    p.close()
                self.packs[n] = Pack(n, k, self.ctas(n))
        torch.cuda.synchronize()
        return plan

    def run(self, requests, realtime=True):
        """Serve `requests` (sorted by arrival); returns per-request records and
        the stream's metrics, as Server.run. realtime=False admits every
        request at t = 0."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        if not all(r.n in self.packs for r in reqs):
            self.prewarm(reqs)
        packs = {n: self.packs[n] for n in sorted({r.n for r in reqs})}
        streams = {n: torch.cuda.Stream() for n in packs}
        mem = {n: [_Member() for _ in range(p.k)] for n, p in packs.items()}
        inflight = {n: None for n in packs}  # (event, CTAs held) of the pack's launch in flight
        pending = {n: [] for n in packs}
        used = 0
        done, nxt = [], 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        while len(done) < len(reqs):
            now = time.perf_counter() - t0
            while nxt < len(reqs) and (not realtime or reqs[nxt].arrival <= now):
                pending[reqs[nxt].n].append(reqs[nxt])
                nxt += 1
            for n, p in packs.items():
                if inflight[n] is not None and inflight[n][0].query():
                    used -= inflight[n][1]
                    inflight[n] = None
                ms = mem[n]
                for m, mb in enumerate(ms):  # retire members whose results have landed
                    if mb.final is not None and mb.final.query():
                        t = time.perf_counter() - t0
                        sl = p.slots[m]
                        r = mb.req
                        rec = {"rid": r.rid, "n": r.n, "arrival": r.arrival, "admitted": mb.admitted, "done": t,
                               "latency": t - (r.arrival if realtime else 0.0), "ctas": p.ctas,
                               "status": int(p.stat_host[5 * m + 4])}
                        if self.keep_results:
                            rec["U"] = sl.U_host.numpy().copy()
                            rec["P"] = sl.P_host.numpy().copy()
                        done.append(rec)
                        ms[m] = _Member()

            # packs without a launch in flight: those with requests under way
            # first (oldest admission first), then those with arrivals only
            def age(n):
                a = [mb.admitted for mb in mem[n] if mb.req is not None and mb.left > 0]
                if a:
                    return (0, min(a))
                return (1, pending[n][0].arrival) if pending[n] else (2, 0.0)

            for n in sorted((n for n in packs if inflight[n] is None), key=age):
                p, ms, st = packs[n], mem[n], streams[n]
                room = (self.capacity - used) // p.ctas
                if room <= 0:
                    continue
                go = [m for m, mb in enumerate(ms) if mb.req is not None and mb.left > 0][:room]
                with torch.cuda.stream(st):
                    for m, mb in enumerate(ms):  # admit into free members while there is room
                        if len(go) >= room or not pending[n]:
                            break
                        if mb.req is None:
                            r = pending[n].pop(0)
                            sl = p.slots[m]
                            sl.U0_host.copy_(torch.from_numpy(r.U0))
                            sl.U[0].copy_(sl.U0_host, non_blocking=True)
                            sl.P[0].zero_()
                            p.stat[5 * m + 4].zero_()
                            mb.req, mb.cur, mb.left = r, 0, r.steps
                            mb.admitted = time.perf_counter() - t0
                            go.append(m)
                if not go:
                    continue
                gs = set(go)
                steps = [min(self.chunk, mb.left) if m in gs else 0 for m, mb in enumerate(ms)]
                p.step([mb.req.dt if mb.req else 1.0 for mb in ms], [mb.req.nu if mb.req else 0.0 for mb in ms],
                       steps, [mb.cur for mb in ms], st)
                ev = torch.cuda.Event()
                ev.record(st)
                inflight[n] = (ev, len(go) * p.ctas)
                used += len(go) * p.ctas
                with torch.cuda.stream(st):
                    for m in go:
                        mb, k = ms[m], steps[m]
                        mb.cur ^= k & 1
                        mb.left -= k
                        if mb.left == 0:
                            sl = p.slots[m]
                            sl.U_host.copy_(sl.U[mb.cur], non_blocking=True)
                            sl.P_host.copy_(sl.P[mb.cur], non_blocking=True)
                            p.stat_host[5 * m:5 * m + 5].copy_(p.stat[5 * m:5 * m + 5], non_blocking=True)
                            mb.final = torch.cuda.Event()
                            mb.final.record(st)
        wall = time.perf_counter() - t0
        lat = np.array([d["latency"] for d in done])
        steps = sum(r.steps for r in reqs)
        return done, {"requests": len(done), "wall_s": wall, "solves_per_s": len(done) / wall,
                      "steps_per_s": steps / wall, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                      "p99_ms": float(np.percentile(lat, 99) * 1e3), "capacity_ctas": self.capacity,
                      "members": {n: p.k for n, p in packs.items()},
                      "share_ctas": {n: p.ctas for n, p in packs.items()}}


def run_plain(requests, server=None):
    """The plain FP64 path: the same requests one after another on the whole
    device (full CTA capacity), each synchronised before the next; returns
    (records, metrics) like Server.run."""
    srv = server or Server()
    srv.warm(sorted({r.n for r in requests}))
    done = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = torch.cuda.current_stream()
    for r in requests:
        slot = srv._take_slot(r.n)
        slot.set_ctas(0)
        slot.U0_host.copy_(torch.from_numpy(r.U0))
        slot.U[0].copy_(slot.U0_host, non_blocking=True)
        slot.P[0].zero_()
        cur = slot.steps(0, r.steps, r.dt, r.nu, st)
        slot.U_host.copy_(slot.U[cur])
        slot.P_host.copy_(slot.P[cur])
        t = time.perf_counter() - t0
        rec = {"rid": r.rid, "n": r.n, "done": t, "latency": t - (done[-1]["done"] if done else 0.0),
               "status": int(slot.solver.status.max().item())}
        if srv.keep_results:
            rec["U"] = slot.U_host.numpy().copy()
            rec["P"] = slot.P_host.numpy().copy()
        done.append(rec)
        srv.pool[r.n].append(slot)
    wall = time.perf_counter() - t0
    steps = sum(r.steps for r in requests)
    lat = np.array([d["latency"] for d in done])
    return done, {"requests": len(done), "wall_s": wall, "solves_per_s": len(done) / wall,
                  "steps_per_s": steps / wall, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                  "p99_ms": float(np.percentile(lat, 99) * 1e3)}
