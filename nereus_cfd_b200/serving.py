"""Batched and served pressure steps through the library's server (include/nereus_b200.h, nereus_b200_server_*):
many independent projections (the tanks of a batch, the requests of a stream) run concurrently on one or more
devices, admitted by a per-device memory budget, each returning like one nereus_b200_project_ex call.

Across processes (torchrun, one process per GPU) the requests are split by the library's deterministic least-loaded
plan (nereus_b200_plan), each rank serves its share on its own device, and the per-rank results are gathered with
torch.distributed (NCCL on GPUs, gloo elsewhere). The solve path itself has no collective.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import capi
from .pressure import MACGrid


@dataclass
class Job:
    """One pressure step: a grid state (fields rewritten in place on completion) and how to solve it."""
    grid: MACGrid
    tol: float = 1e-8
    needs_compat: bool = False
    scheme: int = capi.SCHEME_CHORIN
    p_prev: Optional[np.ndarray] = None
    warm_start: bool = False
    result: Optional[dict] = None
    status: Optional[int] = None
    latency_ms: Optional[float] = None
    device_fields: Optional[dict] = None  # torch CUDA tensors u, v, w, p (, p_prev) when the fields live on the device
    _keep: list = field(default_factory=list, repr=False)

    @property
    def cells(self) -> int:
        return self.grid.grid.cells


def to_device(job: Job, device: int = 0) -> Job:
    """Puts the job's fields on the device (torch tensors): the server then solves them in place, with no host
    copies."""
    import torch

    d = "cuda:%d" % device
    f = {k: torch.from_numpy(np.ascontiguousarray(getattr(job.grid, k), dtype=np.float64)).to(d)
         for k in ("u", "v", "w", "p")}
    if job.p_prev is not None:
        f["p_prev"] = torch.from_numpy(np.ascontiguousarray(job.p_prev, dtype=np.float64)).to(d)
    torch.cuda.synchronize(d)
    job.device_fields = f
    return job


def fetch(job: Job) -> Job:
    """Copies a device job's fields back into its grid arrays."""
    for k in ("u", "v", "w", "p"):
        getattr(job.grid, k)[:] = job.device_fields[k].cpu().numpy()
    return job


def job_from_case(case, tol: Optional[float] = None, types: Optional[np.ndarray] = None) -> Job:
    """A job for one synthetic case: cell labels (on the device unless given), the case's seeded face velocities,
    p = 0 with no prescribed ring values."""
    from . import workloads as W

    g = case.grid
    if types is None:
        types = capi.label_cells(g, case.scene)
    u, v, w = W.face_velocities(g, types, case.seed, case.velocity_rule, case.fp32_velocity)
    m = MACGrid.from_case(case, types, u, v, w)
    return Job(m, tol=case.tol if tol is None else tol, needs_compat=case.needs_compat)


def tank_batch(count: int = 64, n: int = 128, seed: int = 4) -> list:
    """The batch of FLIP-style tanks: ``count`` unit-cube n^3 tanks, liquid where x < a and z < b with a, b ~
    U(0.3, 0.7) drawn per tank from the seed, FP32-rounded liquid-face velocities."""
    from . import workloads as W

    return [W.flip_tank_3d(n, seed=seed + 1000 * t) for t in range(count)]


def request_bytes(job: Job, precision: int = capi.PRECISION_MIXED) -> float:
    g = job.grid.grid
    return capi.load().nereus_b200_request_bytes(g.dim, g.Nx, g.Ny, g.Nz, precision)


def plan(costs: Sequence[float], k: int) -> List[int]:
    """The least-loaded assignment of requests (in order) to k devices or ranks (nereus_b200_plan)."""
    n = len(costs)
    c = np.ascontiguousarray(costs, dtype=np.float64)
    out = (ctypes.c_int * max(n, 1))()
    capi.check(capi.load().nereus_b200_plan(capi.ptr(c), n, k, out))
    return [out[i] for i in range(n)]


class Batch:
    """nereus_b200_batch_*: one pressure step for each of up to ``capacity`` grids of the same shape, advanced by
    the same launches (mixed precision, uniform 3D). Slot i takes jobs[i]; a slot keeps its hierarchy while its
    layout bytes are unchanged. A job's result does not depend on the rest of the batch (the same bits alone or in
    any mix) and agrees with its single-context solve within the tolerance."""

    def __init__(self, capacity: int, device: int = 0, stream: Optional[int] = None, **solver_options):
        self.lib = capi.load()
        self.opts = capi.default_options(device=device, precision=capi.PRECISION_MIXED, **solver_options)
        if stream is not None:
            self.opts.stream = ctypes.c_void_p(stream)
        self.capacity = capacity
        self.h = ctypes.c_void_p()
        capi.check(self.lib.nereus_b200_batch_create(ctypes.byref(self.h), ctypes.byref(self.opts), capacity))
        self._tables = {}

    def set_layout(self, slot: int, grid: MACGrid):
        g = grid.grid
        widths = [np.ascontiguousarray(w) for w in g.width_tables()]
        gaps = [np.ascontiguousarray(x) for x in g.gap_tables()]
        types = np.ascontiguousarray(grid.types, dtype=np.uint8)
        self._tables[slot] = (widths, gaps, types)
        W = (capi._dp * 3)(*[capi.ptr(a) for a in widths])
        G = (capi._dp * 3)(*[capi.ptr(a) for a in gaps])
        capi.check(self.lib.nereus_b200_batch_set_layout(self.h, slot, g.dim, g.Nx, g.Ny, g.Nz,
                                                         capi.ptr(types, capi._u8), W, G, int(g.nonuniform), g.dh))

    def items(self, jobs: Sequence[Job]):
        arr = (capi.BatchItem * len(jobs))()
        for i, j in enumerate(jobs):
            f = j.device_fields
            arr[i].u, arr[i].v, arr[i].w, arr[i].p = (f[k].data_ptr() for k in ("u", "v", "w", "p"))
            arr[i].rho, arr[i].dt = j.grid.rho, j.grid.dt
            arr[i].needs_compat = int(j.needs_compat)
            arr[i].tol = j.tol
        return arr

    def project(self, jobs: Sequence[Job], items=None, allow=(capi.NB_OK, capi.NB_NOT_CONVERGED)):
        """The step of jobs[0 .. n-1] in slots 0 .. n-1 (their layouts set), fields on the device, in place."""
        n = len(jobs)
        res = (capi.Result * n)()
        items = self.items(jobs) if items is None else items
        capi.check(self.lib.nereus_b200_batch_project_device(self.h, n, items, res), allow=allow)
        for j, r in zip(jobs, res):
            j.result = r.as_dict()
            j.status = r.status
        return [r.as_dict() for r in res]

    def info(self) -> dict:
        i = capi.BatchInfo()
        capi.check(self.lib.nereus_b200_batch_info(self.h, ctypes.byref(i)))
        return i.as_dict()

    def close(self):
        if self.h:
            self.lib.nereus_b200_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tune_cache_dump() -> str:
    lib = capi.load()
    n = lib.nereus_b200_tune_cache_dump(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib.nereus_b200_tune_cache_dump(buf, n + 1)
    return buf.value.decode()


def tune_cache_load(text: str) -> int:
    return capi.check(capi.load().nereus_b200_tune_cache_load(text.encode()), allow=range(0, 1 << 30))


class Server:
    """nereus_b200_server_*: submit jobs, poll or wait for them, read the server's statistics."""

    def __init__(self, devices: Sequence[int] = (0,), slots_per_device: int = 4, hbm_budget_gb: float = 150.0,
                 precision: str = "mixed", **solver_options):
        self.lib = capi.load()
        o = capi.ServerOptions()
        self.lib.nereus_b200_default_server_options(ctypes.byref(o))
        self._devs = (ctypes.c_int * len(devices))(*devices)
        o.n_devices = len(devices)
        o.devices = ctypes.cast(self._devs, ctypes.POINTER(ctypes.c_int))
        o.slots_per_device = slots_per_device
        o.hbm_budget_gb = hbm_budget_gb
        o.solver.precision = {"mixed": capi.PRECISION_MIXED, "fp64": capi.PRECISION_FP64}[precision]
        for k, v in solver_options.items():
            setattr(o.solver, k, v)
        self.precision = o.solver.precision
        self.srv = ctypes.c_void_p()
        capi.check(self.lib.nereus_b200_server_create(ctypes.byref(self.srv), ctypes.byref(o)))
        self.jobs = {}

    def submit(self, job: Job) -> int:
        m, g = job.grid, job.grid.grid
        widths = [np.ascontiguousarray(a) for a in g.width_tables()]
        gaps = [np.ascontiguousarray(a) for a in g.gap_tables()]
        types = np.ascontiguousarray(m.types, dtype=np.uint8)
        w = m.w if g.dim == 3 else np.zeros(1)
        r = capi.Request()
        r.dim, r.Nx, r.Ny, r.Nz = g.dim, g.Nx, g.Ny, g.Nz
        r.cell_types = capi.ptr(types, capi._u8)
        for a in range(3):
            r.width[a] = capi.ptr(widths[a])
            r.gap[a] = capi.ptr(gaps[a])
        r.non_uniform, r.dh = int(g.nonuniform), g.dh
        prev = None
        if job.device_fields is not None:
            dp = lambda t: ctypes.cast(t.data_ptr(), capi._dp)
            f = job.device_fields
            r.u, r.v, r.w, r.p = dp(f["u"]), dp(f["v"]), dp(f["w"] if g.dim == 3 else f["u"]), dp(f["p"])
            if "p_prev" in f:
                r.p_prev = dp(f["p_prev"])
            r.fields_on_device = 1
        else:
            r.u, r.v, r.w, r.p = capi.ptr(m.u), capi.ptr(m.v), capi.ptr(w), capi.ptr(m.p)
            if job.p_prev is not None:
                prev = np.ascontiguousarray(job.p_prev, dtype=np.float64)
                r.p_prev = capi.ptr(prev)
        r.scheme, r.needs_compat, r.warm_start = job.scheme, int(job.needs_compat), int(job.warm_start)
        r.rho, r.dt, r.tol = m.rho, m.dt, job.tol
        ticket = ctypes.c_uint64(0)
        capi.check(self.lib.nereus_b200_submit(self.srv, ctypes.byref(r), ctypes.byref(ticket)))
        job._keep = [w, prev]  # the fields must outlive the request
        self.jobs[ticket.value] = (job, time.perf_counter())
        return ticket.value

    def _finish(self, ticket: int, st: int, res: capi.Result):
        job, t0 = self.jobs[ticket]
        job.status = st
        job.result = res.as_dict()
        job.latency_ms = res.latency_ms  # the server's own submission-to-completion time
        return st

    def poll(self, ticket: int) -> int:
        res = capi.Result()
        st = self.lib.nereus_b200_poll(self.srv, ticket, ctypes.byref(res))
        return st if st == capi.NB_BUSY else self._finish(ticket, st, res)

    def wait(self, ticket: int, timeout_s: float = -1.0) -> int:
        res = capi.Result()
        st = self.lib.nereus_b200_wait(self.srv, ticket, timeout_s, ctypes.byref(res))
        return st if st == capi.NB_BUSY else self._finish(ticket, st, res)

    def stats(self) -> dict:
        s = capi.ServerStats()
        capi.check(self.lib.nereus_b200_server_stats(self.srv, ctypes.byref(s)))
        return s.as_dict()

    def reset_stats(self):
        capi.check(self.lib.nereus_b200_server_reset_stats(self.srv))

    def close(self):
        if self.srv:
            self.lib.nereus_b200_server_destroy(self.srv)
            self.srv = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve(jobs: Sequence[Job], server: Server) -> dict:
    """Submits every job, waits for all, and returns the server's statistics (solves/s, p50/p99 latency)."""
    tickets = [server.submit(j) for j in jobs]
    for t in tickets:
        server.wait(t)
    return server.stats()


def run_sharded(items: Sequence, cost: Callable, execute: Callable[[list], dict], dist=None) -> dict:
    """Splits ``items`` (jobs, or cases that ``execute`` turns into jobs) over the ranks of the default process
    group by the least-loaded plan on ``cost(item)``, runs this rank's share with ``execute`` (a list of items ->
    {"seconds": wall seconds, "completed": count, "latencies": [ms, ...]}), and gathers every rank's figures.
    ``seconds`` is the max over ranks, so solves/s = all completions / that time. With no process group it runs
    everything here."""
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist is not None else (0, 1)
    owner = plan([cost(x) for x in items], world)
    mine = [x for x, o in zip(items, owner) if o == rank]
    out = execute(mine)
    local = {"rank": rank, "items": len(mine), "completed": int(out.get("completed", 0)),
             "seconds": float(out.get("seconds", 0.0)), "latencies": list(out.get("latencies", []))}
    if dist is None:
        gathered = [local]
    else:
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
    seconds = max(g["seconds"] for g in gathered)
    lats = sorted(x for g in gathered for x in g["latencies"])
    completed = sum(g["completed"] for g in gathered)

    def pct(q):
        if not lats:
            return None
        k = (len(lats) - 1) * q
        lo, hi = int(k), min(int(k) + 1, len(lats) - 1)
        return lats[lo] + (lats[hi] - lats[lo]) * (k - lo)

    return {"world": world, "completed": completed, "seconds": seconds,
            "solves_per_s": completed / seconds if seconds > 0 else None, "p50_ms": pct(0.5), "p99_ms": pct(0.99),
            "per_rank": [{k: g[k] for k in ("rank", "items", "completed", "seconds")} for g in gathered]}


def serve_jobs(jobs: Sequence[Job], server: Server) -> dict:
    """``execute`` for run_sharded on this rank's device: serve the jobs, report wall seconds from the first
    submission to the last completion, completions, and the server's p50/p99 submission-to-completion latency."""
    server.reset_stats()
    t0 = time.perf_counter()
    tickets = [server.submit(j) for j in jobs]
    for t in tickets:
        server.wait(t)
    seconds = time.perf_counter() - t0
    st = server.stats()
    done = [j for j in jobs if j.status in (capi.NB_OK, capi.NB_NOT_CONVERGED)]
    return {"seconds": seconds, "completed": len(done), "latencies": [j.latency_ms for j in done],
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"]}


# ---------------------------------------------------------------------------------------------------------------------
# a serving trace: requests of mixed dimension, size, mask and spacing arriving as a Poisson process
# ---------------------------------------------------------------------------------------------------------------------
def trace_case(rng, index: int):
    """One request of the trace: 3D with side ~ log-U[32, 256] or 2D with side ~ log-U[64, 1024] (even); mask
    closed box (singular, compatibility on), sphere/disc obstacle with a p = 0 outlet on x = 1, or a free-surface
    tank (liquid where x < a and y or z < b, air elsewhere); uniform, or stretched in x by 1.04 per cell over the
    outer 64 cells of each side."""
    from . import workloads as W

    dim = 3 if rng.random() < 0.5 else 2
    lo, hi = (32, 256) if dim == 3 else (64, 1024)
    n = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi))) / 2.0)) * 2
    mask = ("closed", "obstacle", "free")[int(rng.integers(3))]
    stretched = rng.random() < 0.5
    dom = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    if stretched:
        # a uniform band in the middle, 1.04 growth over the outer 64 cells of each side (width ratio 1.04^64 ~ 12)
        wx = W.band_stretched_widths(n, 1.0, max(2, (n - 128) // 2 * 2), 0.5, 1.04)
        ws = [wx, np.full(n, 1.0 / n)] + ([np.full(n, 1.0 / n)] if dim == 3 else [])
        g = W.stretched_grid(dim, dom, ws)
    else:
        g = W.uniform_grid(dim, dom, n)
    compat, rule = False, "solid"
    if mask == "closed":
        sc, compat = W.walls_scene(dim), True
    elif mask == "obstacle":
        sph = W.Region(W.REGION_SOLID, W.PRIM_SPHERE, (0.5, 0.5, 0.5), radius=0.15)
        sc = W.walls_scene(dim, outlet_face=1, regions=[sph])
    else:
        a, b = rng.uniform(0.3, 0.7, 2)
        air = W.Region(W.REGION_EMPTY, W.PRIM_BOX, (-1.0, -1.0, -1.0), (2.0, 2.0, 2.0))
        top = (a, 2.0, b) if dim == 3 else (a, b, 2.0)
        liquid = W.Region(W.REGION_FLUID, W.PRIM_BOX, (-1.0, -1.0, -1.0), top)
        sc, rule = W.walls_scene(dim, regions=[air, liquid]), "liquid"
    name = "trace%d_%dd_%d_%s_%s" % (index, dim, n, mask, "stretched" if stretched else "uniform")
    return W.Case(name, g, sc, int(rng.integers(1 << 31)), needs_compat=compat, velocity_rule=rule)


def device_job(case, device: int = 0, tol: float = 1e-8, types: Optional[np.ndarray] = None, dtypes=None) -> Job:
    """A job whose fields are drawn on the device: labels by the library (or the given host `types` and their device
    copy `dtypes`), N(0,1) face velocities from a torch generator seeded by the case, zeroed by the case's rule
    (face_velocities' rules), p = 0."""
    import torch

    from . import workloads as W

    g = case.grid
    if types is None:
        types = capi.label_cells(g, case.scene)
    d = "cuda:%d" % device
    t = dtypes.reshape(g.shape) if dtypes is not None else torch.from_numpy(types.reshape(g.shape)).to(d)
    gen = torch.Generator(device=d)
    gen.manual_seed(case.seed)
    fields = {}
    comps = 3 if g.dim == 3 else 2
    for c in range(comps):
        shape = [g.u_shape(), g.v_shape(), g.w_shape()][c]
        vals = torch.randn(shape, generator=gen, device=d, dtype=torch.float64)
        ax = [1, 0, 2][c]
        pad = [0, 0, 0, 0, 0, 0]  # last dim first
        pad[2 * (2 - ax)] = pad[2 * (2 - ax) + 1] = 1
        tp = torch.nn.functional.pad(t, pad, value=W.SOLID)
        a, b = tp.narrow(ax, 0, tp.shape[ax] - 1), tp.narrow(ax, 1, tp.shape[ax] - 1)
        keep = (a != W.SOLID) & (b != W.SOLID)
        if case.velocity_rule == "liquid":
            keep &= (a == W.FLUID) | (b == W.FLUID)
        fields["uvw"[c]] = torch.where(keep, vals, torch.zeros_like(vals)).reshape(-1).contiguous()
    if comps == 2:
        fields["w"] = torch.zeros(1, dtype=torch.float64, device=d)
    fields["p"] = torch.zeros(g.cells, dtype=torch.float64, device=d)
    m = MACGrid(g, types, np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), case.rho, case.dt)
    job = Job(m, tol=tol, needs_compat=case.needs_compat)
    job.device_fields = fields
    torch.cuda.current_stream(d).synchronize()  # the fields are written before any slot's stream reads them
    return job


def trace_labels(cases: Sequence, device: int = 0):
    """The cell types of every case, computed once by the library: host arrays and their device copies."""
    import torch

    host, dev = [], []
    for c in cases:
        t = capi.label_cells(c.grid, c.scene)
        host.append(t)
        dev.append(torch.from_numpy(t).to("cuda:%d" % device))
    torch.cuda.synchronize(device)
    return host, dev


_PRODUCERS = {}  # device -> (the job producers' stream, bytes reserved in its cache)


class JobStream:
    """The device jobs of a list of cases, made by a background thread a bounded number ahead of use (so a long
    trace never holds more than `ahead` unsubmitted requests' fields on the device). Iterate to take them in order.
    labels: (host, device) cell types of the cases (trace_labels), else each job labels its case."""

    def __init__(self, cases: Sequence, device: int = 0, tol: float = 1e-8, ahead: int = 16, labels=None):
        import queue
        import threading

        # device memory for the fields and their temporaries (about 48 B per cell), reserved up front in the
        # producer stream's cache: a cudaMalloc while solves run holds up every thread on the device (measured: tens
        # to hundreds of ms), so making a request must not call it
        sizes = sorted((c.grid.cells for c in cases), reverse=True)[: ahead + 4]
        reserve = 48 * sum(sizes)

        self.q = queue.Queue(maxsize=max(1, ahead))
        self.n = len(cases)
        self.error = None
        self.make_seconds = 0.0  # time the producer spent making jobs (not waiting for room)

        def produce():
            import torch

            torch.cuda.set_device(device)
            # a high-priority stream, one per device for every stream of jobs (torch caches memory per stream, so the
            # reservation below serves later streams too): the fields are drawn while the solves keep the GPU busy
            stream, held = _PRODUCERS.get(device, (None, 0))
            if stream is None:
                lo, hi = torch.cuda.Stream.priority_range() if hasattr(torch.cuda.Stream, "priority_range") else (0, -1)
                stream = torch.cuda.Stream(device=device, priority=min(lo, hi))
            try:
                with torch.cuda.stream(stream):
                    if reserve > held:
                        block = torch.empty(reserve, dtype=torch.uint8, device="cuda:%d" % device)
                        del block  # stays in this stream's cache; the requests' tensors are carved out of it
                    _PRODUCERS[device] = (stream, max(held, reserve))
                    for k, c in enumerate(cases):
                        t = time.perf_counter()
                        j = device_job(c, device, tol, *((labels[0][k], labels[1][k]) if labels else ()))
                        self.make_seconds += time.perf_counter() - t
                        self.q.put(j)
            except Exception as e:  # reported to the consumer
                self.error = e
                self.q.put(None)

        self.t = threading.Thread(target=produce, daemon=True)
        self.t.start()

    def __iter__(self):
        for _ in range(self.n):
            j = self.q.get()
            if j is None:
                raise RuntimeError("making a trace request failed: %s" % self.error)
            yield j


def stream_serve(server: Server, cases: Sequence, device: int = 0, tol: float = 1e-8, rate: Optional[float] = None,
                 seed: int = 0, inflight: int = 16, ahead: int = 16, labels=None) -> dict:
    """Serves the cases' requests as they are made (JobStream): with `rate`, submitted at Poisson arrival times of
    that rate (per second); without, as a closed loop keeping `inflight` requests submitted. A completed request's
    device fields are dropped at once. Latency: the server's own, from submission to completion, and, under Poisson
    arrivals, from the arrival time (the two differ when a request was made after its arrival was due)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, len(cases)) if rate else None
    server.reset_stats()
    out = {}  # ticket -> (job, submitted at, due at)
    lat, lat_due, iters = [], [], []
    failed = 0

    def reap(block: bool):
        nonlocal failed
        if block and out:
            server.wait(next(iter(out)), 0.002)  # blocks in the library (the GIL released) up to 2 ms
        while out:
            done = []
            for t, (j, ts, td) in out.items():
                st = server.poll(t)
                if st == capi.NB_BUSY:
                    continue
                done.append(t)
                if st in (capi.NB_OK, capi.NB_NOT_CONVERGED):
                    lat.append(j.latency_ms)
                    lat_due.append(1e3 * (ts - td) + j.latency_ms)
                    iters.append(j.result["iters_inner"] if j.result else 0)
                else:
                    failed += 1
                j.device_fields = None
            for t in done:
                del out[t]
            if not block or done:
                return
            time.sleep(0.0002)

    stream = JobStream(cases, device, tol, ahead, labels)
    t0 = time.perf_counter()
    due = t0
    for k, j in enumerate(stream):
        if gaps is not None:
            due += gaps[k]
            while time.perf_counter() < due:
                reap(False)
                time.sleep(min(0.0005, max(0.0, due - time.perf_counter())))
        else:
            while len(out) >= inflight:
                reap(True)
            due = time.perf_counter()
        ts = time.perf_counter()
        out[server.submit(j)] = (j, ts, due)
        reap(False)
    while out:
        reap(True)
    seconds = time.perf_counter() - t0

    def pct(xs, q):
        xs = sorted(xs)
        if not xs:
            return None
        kk = (len(xs) - 1) * q
        lo, hi = int(kk), min(int(kk) + 1, len(xs) - 1)
        return round(xs[lo] + (xs[hi] - xs[lo]) * (kk - lo), 3)

    r = {"requests": len(cases), "completed": len(lat), "failed": failed, "seconds": round(seconds, 4),
         "make_seconds": round(stream.make_seconds, 3),
         "solves_per_s": round(len(lat) / seconds, 3), "p50_ms": pct(lat, 0.5), "p99_ms": pct(lat, 0.99),
         "iters_inner_mean": round(float(np.mean(iters)), 2) if iters else None}
    st = server.stats()
    r["slot_layout_s"], r["slot_project_s"] = round(st["layout_s"], 3), round(st["project_s"], 3)
    if rate:
        r["rate_per_s"] = round(rate, 3)
        r["p50_ms_from_arrival"], r["p99_ms_from_arrival"] = pct(lat_due, 0.5), pct(lat_due, 0.99)
    return r


def run_trace(server: Server, jobs: Sequence[Job], rate: float, seed: int = 0) -> dict:
    """Submits the jobs at Poisson arrival times of the given rate (per second) and waits for all. Latency is the
    server's own, from a request's submission (its arrival) to its completion."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, len(jobs))
    server.reset_stats()
    t0 = time.perf_counter()
    due = t0
    tickets = []
    for j, gap in zip(jobs, gaps):
        due += gap
        while time.perf_counter() < due:
            time.sleep(min(0.0005, max(0.0, due - time.perf_counter())))
        j.latency_ms = None
        tickets.append(server.submit(j))
    for t in tickets:
        server.wait(t)
    seconds = time.perf_counter() - t0
    st = server.stats()
    return {"rate_per_s": round(rate, 3), "requests": len(jobs), "completed": st["completed"],
            "failed": st["failed"], "seconds": round(seconds, 4), "solves_per_s": round(st["completed"] / seconds, 3),
            "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3)}
