"""Benchmark of the B200 pressure projection: solves/s and p50/p99 latency at a 1e-8 relative residual.

Workload (the configuration the metric is quoted on, one GPU): 3D 256^3 unit cube, uniform, a voxelised solid sphere
at (0.5, 0.5, 0.5) radius 0.15 sampled at cell centres, no-slip walls, a p = 0 pressure outlet on x = 1; face
velocities N(0,1) FP64 from a seeded SplitMix64/Box-Muller generator (synthetic data), zeroed on solid faces.
A step is one pressure projection of that field: divergence/right-hand side, FP32 MG-PCG inside FP64 iterative
refinement to ||b - A x|| / ||b|| <= 1e-8, level, scatter, ring, velocity correction. Each step restores the
unprojected fields by a device copy first (inside the timed region), so every step solves the full problem; the
552 MB of fields read per step are larger than the 126 MB L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With N > 1 (torchrun, one rank per GPU) every rank projects its own field (seeded per rank): weak scaling, no
collective on the data path; the timing is the max over ranks.

The JSON line also carries the plain single-solve FP64 MG-PCG form on the same workload, the roofline of the
dominant kernel (CUDA events around its launches over the timed region, algorithmic bytes per launch), the end-to-end
number through the C ABI with host buffers, the reference's CPU path timed on this host, clocks sampled during the
timed region and the count of this library's kernel launches.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s, p50/p99 latency at 1e-8 rel residual: batched mixed vs plain FP64"
TOL = 1e-8


def percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = (len(xs) - 1) * q
    lo, hi = int(k), min(int(k) + 1, len(xs) - 1)
    return xs[lo] + (xs[hi] - xs[lo]) * (k - lo)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary (profiles/*.md line
    'traffic_bytes_per_launch <kernel> <bytes> <cells>'), scaled to the bench's cell count by the caller."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for fn in sorted(os.listdir(d)):
        if not fn.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(d, fn)):
            parts = line.strip().strip("`").split()
            if len(parts) == 4 and parts[0] == "traffic_bytes_per_launch" and parts[1] == kernel:
                return float(parts[2]), float(parts[3])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, val in zip(names[1:], p[5:9]):
                if val.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------------------------------------
# the workload
# ---------------------------------------------------------------------------------------------------------------------
def make_workload(n: int, seed: int):
    from nereus_cfd_b200 import capi, workloads as W

    case = W.sphere_outlet_3d(n, seed=seed)
    types = capi.label_cells(case.grid, case.scene)
    u, v, w = W.face_velocities(case.grid, types, case.seed)
    return case, types, u, v, w


def run_b200(args, rank, world, dist):
    import torch

    from nereus_cfd_b200 import capi
    from nereus_cfd_b200.pressure import MACGrid, PressureSolver

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    lib = capi.load()
    case, types, u, v, w = make_workload(args.size, seed=2 + 1000 * rank)
    g = case.grid
    stream = torch.cuda.current_stream()
    td = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to("cuda")
    U0, V0, W0 = td(u), td(v), td(w)
    P0 = torch.zeros(g.cells, dtype=torch.float64, device="cuda")
    U, V, Wf, P = U0.clone(), V0.clone(), W0.clone(), P0.clone()
    mac = MACGrid.from_case(case, types, u, v, w)

    def project_steps(solver, steps, times=None, start=None):
        res = capi.Result()
        for _ in range(steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            U.copy_(U0); V.copy_(V0); Wf.copy_(W0); P.copy_(P0)
            st = lib.nereus_b200_project_device(solver.ctx, U.data_ptr(), V.data_ptr(), Wf.data_ptr(),
                                                P.data_ptr(), case.rho, case.dt, 0, TOL, ctypes.byref(res))
            capi.check(st)
            e1.record(stream)
            if times is not None:
                times.append((e0, e1))
        return res

    def timed(solver, steps, warmup, profile_mask=0, clocks=False):
        # the mask is set before the warm-up, so the captured iteration graph (with its event nodes) is built there;
        # setting it again clears the totals only
        capi.check(lib.nereus_b200_profile_enable(solver.ctx, profile_mask))
        project_steps(solver, warmup)
        capi.check(lib.nereus_b200_profile_enable(solver.ctx, profile_mask))
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(dev) if clocks else None
        if sampler:
            sampler.start()
        launches0 = lib.nereus_b200_kernel_launches()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        times = []
        start.record(stream)
        res = project_steps(solver, steps, times)
        end.record(stream)
        torch.cuda.synchronize()
        launches = lib.nereus_b200_kernel_launches() - launches0
        clk = sampler.stop() if sampler else None
        if dist:
            dist.barrier()
        total_ms = start.elapsed_time(end)
        lat = [a.elapsed_time(b) for a, b in times]
        prof = capi.profile_read(lib, solver.ctx) if profile_mask else {}
        capi.check(lib.nereus_b200_profile_enable(solver.ctx, 0))
        return total_ms, lat, res, launches, clk, prof

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- the chosen form: FP32 MG-PCG inside FP64 refinement ----
    mixed = PressureSolver("mixed", device=dev, stream=stream.cuda_stream, **args.solver_opts)
    mixed.InitializePressureSolver(mac)
    # the headline: no timing events inside the solve
    total_ms, lat, res, launches, clk, _ = timed(mixed, args.steps, args.warmup, clocks=True)
    total_ms = max_over_ranks(total_ms)
    value = world * args.steps / (total_ms / 1e3)
    # the breakdown: events around every kernel of the solve (they cost some time of their own, so the shares come
    # from this pass and the headline from the one above)
    _, _, _, _, _, prof = timed(mixed, args.steps, args.warmup, profile_mask=(1 << len(capi.KERNEL_NAMES)) - 1)

    # ---- roofline of the dominant kernel (largest summed device time), timed alone: events around its launches only
    peak, peak_kind = measured_peaks()
    roof = None
    if prof:
        name, _ = max(((k, v) for k, v in prof.items() if v[2] > 0), key=lambda kv: kv[1][1])
        kid = capi.KERNEL_NAMES.index(name)
        _, _, _, _, _, prof1 = timed(mixed, args.steps, args.warmup, profile_mask=1 << kid)
        cnt, ms, bpl = prof1[name]
        per_launch_s = ms / cnt / 1e3
        achieved = bpl / per_launch_s / 1e9
        tr = ncu_traffic(name)
        traffic = None
        if tr:
            traffic = tr[0] * (g.cells / tr[1])
        roof = {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": bpl, "launches": cnt, "avg_launch_us": round(per_launch_s * 1e6, 2),
                "share_of_timed_region": round(ms / max(sum(x[1] for x in prof.values()), 1e-9), 4),
                "kernels": {k: {"launches": v[0], "ms": round(v[1], 3),
                                "GB/s": round(v[2] / (v[1] / v[0] / 1e3) / 1e9, 1) if v[2] else None}
                            for k, v in prof.items()}}
    mixed_res = res.as_dict()
    mixed.DestroyPressureSolver()

    # ---- the plain single-solve FP64 MG-PCG form on the same workload ----
    fp64 = None
    if not args.no_fp64:
        plain = PressureSolver("fp64", device=dev, stream=stream.cuda_stream, **args.solver_opts)
        plain.InitializePressureSolver(mac)
        ksteps = max(3, min(args.steps, args.fp64_steps))
        t64, lat64, r64, _, _, _ = timed(plain, ksteps, 1)
        t64 = max_over_ranks(t64)
        v64 = world * ksteps / (t64 / 1e3)
        fp64 = {"value": round(v64, 3), "unit": "solves/s", "steps": ksteps,
                "p50_ms": round(percentile(lat64, 0.5), 3), "p99_ms": round(percentile(lat64, 0.99), 3),
                "iters": r64.iters_inner, "rel_res": r64.rel_res, "speedup_mixed_over_fp64": round(value / v64, 3)}
        plain.DestroyPressureSolver()

    # ---- end to end through the C ABI with host buffers (pinned), H2D + D2H inside every step ----
    e2e = None
    if not args.no_e2e:
        s = PressureSolver("mixed", device=dev, **args.solver_opts)
        s.InitializePressureSolver(mac)
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).pin_memory().numpy()
        hu0, hv0, hw0 = pin(u), pin(v), pin(w)
        hp0 = np.zeros(g.cells)
        hu, hv, hw, hp = pin(u), pin(v), pin(w), pin(hp0)
        res = capi.Result()

        def call():
            np.copyto(hu, hu0); np.copyto(hv, hv0); np.copyto(hw, hw0); np.copyto(hp, hp0)
            t0 = time.perf_counter()
            capi.check(lib.nereus_b200_project(s.ctx, capi.ptr(hu), capi.ptr(hv), capi.ptr(hw), capi.ptr(hp),
                                               case.rho, case.dt, 0, 0, TOL, ctypes.byref(res)))
            return time.perf_counter() - t0

        for _ in range(max(1, args.warmup)):
            call()
        ke = max(3, min(args.steps, args.e2e_steps))
        if dist:
            dist.barrier()
        ts = [call() for _ in range(ke)]
        tot = max_over_ranks(sum(ts))
        nbytes = 8 * (hu.size + hv.size + hw.size + hp.size)
        e2e = {"value": round(world * ke / tot, 3), "unit": "solves/s", "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "steps": ke, "p50_ms": round(1e3 * percentile(ts, 0.5), 3),
               "p99_ms": round(1e3 * percentile(ts, 0.99), 3), "api": "nereus_b200_project (host buffers)"}
        s.DestroyPressureSolver()

    stretched = run_stretched(args, dev) if args.stretched_steps > 0 and world == 1 else None
    tanks = run_tanks(args, rank, world, dist, dev) if args.tanks > 0 else None
    trace = run_trace(args, dev) if args.trace > 0 and world == 1 else None
    relabel = None
    if args.relabel_steps > 0 and world == 1:
        try:
            relabel = run_relabel(args, dev)
        except Exception as e:  # a side measurement: reported, never fatal to the headline line
            relabel = {"unavailable": "%s: %s" % (type(e).__name__, str(e)[:300])}

    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 MG-PCG in f64 refinement", "data": "synthetic",
        "config": {"workload": "sphere_outlet_3d_%d" % args.size,
                   "grid": "%dx%dx%d cells incl. ring, uniform, unit cube" % (g.Nx, g.Ny, g.Nz),
                   "unknowns": mixed_res["n"], "tol": TOL, "precision": "mixed",
                   "parallelism": "replicas x%d" % world, "levels": mixed_res["levels"],
                   "l2": "inputs larger than L2 (552 MB of fields per step), restored by device copy in each step"},
        "latency_ms": {"p50": round(percentile(lat, 0.5), 3), "p99": round(percentile(lat, 0.99), 3)},
        "solve": {k: mixed_res[k] for k in ("iters_outer", "iters_inner", "rel_res", "max_div", "status")},
        "fp64_plain": fp64, "roofline": roof, "e2e": e2e, "clocks": clk, "gpu_launches": int(launches),
        "stretched_cylinder": stretched, "batched_tanks": tanks, "serving_trace": trace, "flip_relabel": relabel,
    }
    return out


def run_trace(args, dev):
    """The served form: `trace` requests of mixed dimension (3D side log-U[32, 256], 2D side log-U[64, 1024]), mask
    (closed, obstacle + outlet, free surface) and spacing (uniform, 1.04-stretched), fields drawn on the device, each
    to 1e-8. A closed loop (all submitted at once) gives the capacity; Poisson arrivals at 0.5x and 0.9x of it give
    p50/p99 latency from arrival to completion; the first `trace_fp64` requests are also solved one at a time in plain
    FP64 on the device (the one-at-a-time path)."""
    import torch

    from nereus_cfd_b200 import capi, serving
    from nereus_cfd_b200.pressure import PressureSolver

    rng = np.random.default_rng(5)
    cases = [serving.trace_case(rng, i) for i in range(args.trace)]
    fresh = lambda cs: [serving.device_job(c, dev, TOL) for c in cs]
    out = {"requests": len(cases), "slots_per_device": args.slots, "hbm_budget_gb": 150.0,
           "mix": {"3d": sum(c.grid.dim == 3 for c in cases), "2d": sum(c.grid.dim == 2 for c in cases),
                   "stretched": sum(c.grid.nonuniform for c in cases)}}
    with serving.Server(devices=(dev,), slots_per_device=args.slots, hbm_budget_gb=150.0, **args.solver_opts) as srv:
        # warm-up: the largest requests first, so that every slot's device arrays hold the trace's biggest shapes
        biggest = sorted(cases, key=lambda c: -c.grid.cells)[: args.slots]
        serving.serve_jobs(fresh(biggest), srv)
        closed = serving.serve_jobs(fresh(cases), srv)
        cap = closed["completed"] / closed["seconds"]
        out["closed_loop"] = {"solves_per_s": round(cap, 3), "seconds": round(closed["seconds"], 4),
                              "p50_ms": round(closed["p50_ms"], 3), "p99_ms": round(closed["p99_ms"], 3)}
        out["poisson"] = [serving.run_trace(srv, fresh(cases), f * cap, seed=11 + k)
                          for k, f in enumerate((0.5, 0.9))]
        # the first `trace_fp64` requests served again (the server as warmed above) ...
        k = min(args.trace_fp64, len(cases))
        same = serving.serve_jobs(fresh(cases[:k]), srv)
    # ... and one at a time in plain FP64, its context warmed the same way (on the largest request first)
    sample = fresh(cases[:k])
    s = PressureSolver("fp64", device=dev, **args.solver_opts)
    lib = capi.load()

    def one(j):
        s.EnsureSystem(j.grid)
        f, res = j.device_fields, capi.Result()
        capi.check(lib.nereus_b200_project_device(s.ctx, f["u"].data_ptr(), f["v"].data_ptr(), f["w"].data_ptr(),
                                                  f["p"].data_ptr(), j.grid.rho, j.grid.dt, int(j.needs_compat), TOL,
                                                  ctypes.byref(res)), allow=(0, 1))

    warm = fresh([max(cases[:k], key=lambda c: c.grid.cells)])[0]
    s.InitializePressureSolver(warm.grid)
    one(warm)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for j in sample:
        one(j)
    torch.cuda.synchronize()
    fp64_rate = k / (time.perf_counter() - t0)
    s.DestroyPressureSolver()
    out["fp64_one_at_a_time"] = {"value": round(fp64_rate, 3), "unit": "solves/s", "requests": k}
    out["served_same_requests"] = {"value": round(same["completed"] / same["seconds"], 3), "unit": "solves/s",
                                   "requests": k}
    out["speedup_over_fp64_one_at_a_time"] = round(same["completed"] / same["seconds"] / fp64_rate, 3)
    out["timing"] = "host wall clock; latency from submission (arrival) to completion"
    return out


def run_stretched(args, dev):
    """The stretched workload: 192x128x128 on [0,2.2]x[0,0.41]^2, widths x 1.04 per cell away from a 24-cell band
    at x = 0.5, a solid cylinder along z, inflow at x = 0, p = 0 outlet at x = 2.2, seeded N(0,1) faces; mixed and
    plain FP64 to 1e-8, fields device-resident and restored each step, CUDA events."""
    import torch

    from nereus_cfd_b200 import capi, workloads as W
    from nereus_cfd_b200.pressure import MACGrid, PressureSolver

    lib = capi.load()
    case = W.stretched_cylinder_3d(192, 128, 128, seed=3)
    types = capi.label_cells(case.grid, case.scene)
    u, v, w = W.face_velocities(case.grid, types, case.seed)
    td = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to("cuda")
    orig = [td(u), td(v), td(w), torch.zeros(case.grid.cells, dtype=torch.float64, device="cuda")]
    work = [t.clone() for t in orig]
    out = {"workload": "stretched_cylinder_192x128x128", "unknowns": None}
    for prec in ("mixed", "fp64"):
        s = PressureSolver(prec, device=dev, **args.solver_opts)
        s.InitializePressureSolver(MACGrid.from_case(case, types, u, v, w))
        res = capi.Result()
        evs = []
        for k in range(3 + args.stretched_steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for x, y in zip(work, orig):
                x.copy_(y)
            capi.check(lib.nereus_b200_project_device(s.ctx, *[t.data_ptr() for t in work], case.rho, case.dt, 0,
                                                      TOL, ctypes.byref(res)), allow=(0, 1))
            b.record()
            if k >= 3:
                evs.append((a, b))
        torch.cuda.synchronize()
        ms = [a.elapsed_time(b) for a, b in evs]
        out[prec] = {"value": round(1e3 / statistics.mean(ms), 3), "unit": "solves/s",
                     "p50_ms": round(percentile(ms, 0.5), 3), "iters_inner": res.iters_inner,
                     "iters_outer": res.iters_outer, "rel_res": res.rel_res, "steps": len(ms)}
        out["unknowns"] = res.n
        s.DestroyPressureSolver()
    out["speedup_mixed_over_fp64"] = round(out["mixed"]["value"] / out["fp64"]["value"], 3)
    return out


def run_relabel(args, dev):
    """FLIP's re-labelling from particles (nereus_b200_update_fluid_cells_device; FLIP3D::UpdateFluidCells): the
    free-surface tank at 256^3 (liquid where x < 0.5 and z < 0.5), 8 particles per liquid cell seeded cell by cell
    (the reference's seeding order) with 3% of the liquid cells left empty, positions as (x, y, z) rows of float64
    and as the reference's 7-double Particle rows. The call resets the labels itself, so repeated steps start from
    the previous step's labels exactly as the reference's do. CUDA events on the launching stream; the position rows
    (805 MB) are larger than L2. The host form (host arrays in, labels out) is timed by wall clock, and the oracle's
    serial restatement on one host core is the CPU baseline."""
    import torch

    from nereus_cfd_b200 import capi, workloads as W

    lib = capi.load()
    n = args.relabel_size
    case = W.flip_tank_3d(n=n, seed=4, a=0.5, b=0.5)
    g = case.grid
    types = capi.label_cells(g, case.scene)
    org = [ax.face[0] for ax in g.axes]
    gen = torch.Generator(device="cuda")
    gen.manual_seed(4)
    liquid = torch.nonzero(torch.from_numpy(types.reshape(g.shape) == W.FLUID).to("cuda"))  # (i, j, k) in order
    keep = torch.rand(liquid.shape[0], device="cuda", generator=gen, dtype=torch.float64) >= 0.03
    cells = liquid[keep].repeat_interleave(8, dim=0)
    faces = [torch.from_numpy(ax.face).to("cuda") for ax in g.axes]
    jit = torch.rand(cells.shape[0], 3, device="cuda", generator=gen, dtype=torch.float64)
    rows = torch.stack([faces[0][cells[:, 1]], faces[1][cells[:, 0]], faces[2][cells[:, 2]]], dim=1) + g.dh * jit
    rows = rows.contiguous()
    del cells, jit
    count = rows.shape[0]
    t = torch.from_numpy(types).to("cuda")
    sb = lib.nereus_b200_update_fluid_cells_scratch_bytes(3, g.Nx, g.Ny, g.Nz)
    scratch = torch.zeros(sb // 4 + 1, dtype=torch.int32, device="cuda")
    skipped = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = torch.cuda.current_stream()

    def step(px, py, pz, stride):
        capi.check(lib.nereus_b200_update_fluid_cells_device(
            dev, 3, g.Nx, g.Ny, g.Nz, org[0], org[1], org[2], g.dh, ctypes.c_void_p(px), ctypes.c_void_p(py),
            ctypes.c_void_p(pz), count, stride, ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(scratch.data_ptr()),
            sb, ctypes.c_void_p(skipped.data_ptr()), ctypes.c_void_p(st.cuda_stream)))

    def timed(px, py, pz, stride):
        for _ in range(3):
            step(px, py, pz, stride)
        evs = []
        l0 = lib.nereus_b200_kernel_launches()
        for _ in range(args.relabel_steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            step(px, py, pz, stride)
            b.record(st)
            evs.append((a, b))
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs], lib.nereus_b200_kernel_launches() - l0

    base = rows.data_ptr()
    ms, launches = timed(base, base + 8, base + 16, 3)
    peak, peak_kind = measured_peaks()
    algo = 24 * count + 5 * g.cells  # positions; labels: reset r+w, fill r, finish r+w
    med = statistics.median(ms)
    out = {"workload": "flip_tank_3d_%d, 8 particles per liquid cell" % n, "particles": count, "cells": g.cells,
           "value": round(count / med / 1e3, 1), "unit": "M particles/s", "ms": round(med, 4),
           "steps": len(ms), "gpu_launches": int(launches), "skipped": int(skipped.item()),
           "roofline": {"bound": "hbm", "achieved": round(algo / med / 1e6, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(algo / med / 1e6 / peak, 3), "peak_kind": peak_kind,
                        "traffic": None, "algorithmic_bytes": int(algo),
                        "bytes_per_unit": "24 B per particle (x, y, z) + 5 B per cell (labels reset, read, finished)"}}
    tr = ncu_traffic("relabel_call")  # DRAM bytes of one call from the committed ncu summary, scaled by cells
    if tr is not None:
        out["roofline"]["traffic"] = int(tr[0] * g.cells / tr[1])
    # the reference's own Particle layout: 7 doubles a particle, x at the second
    aos = torch.zeros(count, 7, dtype=torch.float64, device="cuda")
    aos[:, 1:4] = rows
    ab = aos.data_ptr()
    ms7, _ = timed(ab + 8, ab + 16, ab + 24, 7)
    out["particle_rows_7"] = {"value": round(count / statistics.median(ms7) / 1e3, 1), "unit": "M particles/s",
                              "ms": round(statistics.median(ms7), 4)}
    del aos
    # host form end to end: host positions and labels in, labels out
    hx = rows.cpu().numpy()
    ts = []
    for _ in range(2):
        t0 = time.perf_counter()
        capi.update_fluid_cells(g, types, hx, org)
        ts.append(time.perf_counter() - t0)
    out["e2e"] = {"value": round(count / min(ts) / 1e6, 1), "unit": "M particles/s", "ms": round(1e3 * min(ts), 2),
                  "api": "nereus_b200_update_fluid_cells (host arrays)", "h2d_bytes_per_step": 24 * count + g.cells,
                  "d2h_bytes_per_step": g.cells + 8}
    if not args.no_cpu_baseline:
        from oracle import cpu

        t0 = time.perf_counter()
        cpu.update_fluid_cells(g, types, hx, org)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(count / dt / 1e6, 2), "unit": "M particles/s", "cores": 1,
                               "kind": "port", "sample": "the whole cloud, oracle/pressure_oracle.c serial"}
    return out


def run_tanks(args, rank, world, dist, dev):
    """The batched form: `tanks` FLIP-style n^3 tanks (liquid where x < a, z < b; a, b ~ U(0.3, 0.7) per tank),
    each one pressure step to 1e-8 through the server (`slots` concurrent solves on this rank's device; the tanks'
    fields resident on the device as in a simulation step, each request bringing its own cell labels), split over the
    ranks by the least-loaded plan; against the same tanks solved one at a time in plain FP64 on the device. Wall
    clock from the first submission to the last completion, max over ranks."""
    import copy

    from nereus_cfd_b200 import capi, serving
    from nereus_cfd_b200.pressure import PressureSolver

    cases = serving.tank_batch(args.tanks, args.tank_size)
    summary = {}

    import torch

    def execute(mine):
        jobs = [serving.to_device(serving.job_from_case(c, tol=TOL), dev) for c in mine]
        if not jobs:
            return {"seconds": 0.0, "completed": 0, "latencies": []}
        with serving.Server(devices=(dev,), slots_per_device=args.slots, **args.solver_opts) as srv:
            warm = [copy.deepcopy(j) for j in jobs[: args.slots]]
            serving.serve_jobs(warm, srv)  # each slot's context, graphs and buffers
            out = serving.serve_jobs(jobs, srv)
        out["iters_inner"] = [j.result["iters_inner"] for j in jobs if j.result]
        # one at a time in plain FP64 on a sample of the same tanks, fields on the device likewise
        sample = [serving.to_device(serving.job_from_case(c, tol=TOL), dev) for c in mine[: args.fp64_tanks]]
        s = PressureSolver("fp64", device=dev, **args.solver_opts)
        lib = capi.load()

        def one(j):
            s.EnsureSystem(j.grid)
            f, res = j.device_fields, capi.Result()
            capi.check(lib.nereus_b200_project_device(s.ctx, f["u"].data_ptr(), f["v"].data_ptr(), f["w"].data_ptr(),
                                                      f["p"].data_ptr(), j.grid.rho, j.grid.dt, 0, TOL,
                                                      ctypes.byref(res)), allow=(0, 1))

        s.InitializePressureSolver(sample[0].grid)
        one(copy.deepcopy(sample[0]))  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for j in sample:
            one(j)
        torch.cuda.synchronize()
        out["fp64_seconds_each"] = (time.perf_counter() - t0) / len(sample)
        s.DestroyPressureSolver()
        summary.update(out)
        return out

    res = serving.run_sharded(cases, lambda c: c.grid.cells, execute, dist)
    fp64_each = summary.get("fp64_seconds_each")
    if dist:
        vals = [None] * world
        dist.all_gather_object(vals, fp64_each)
        fp64_each = max(v for v in vals if v is not None)
    fp64_rate = world / fp64_each if fp64_each else None
    its = summary.get("iters_inner", [])
    return {"workload": "flip_tanks_%dx%d^3" % (args.tanks, args.tank_size), "tanks": args.tanks,
            "slots_per_device": args.slots, "value": round(res["solves_per_s"], 3), "unit": "solves/s",
            "p50_ms": round(res["p50_ms"], 3), "p99_ms": round(res["p99_ms"], 3), "seconds": round(res["seconds"], 4),
            "scaling": "strong", "iters_inner_rank0": [int(min(its)), int(max(its))] if its else None,
            "fp64_one_at_a_time": {"value": round(fp64_rate, 3) if fp64_rate else None, "unit": "solves/s",
                                   "sample_tanks": args.fp64_tanks},
            "speedup_over_fp64_one_at_a_time": round(res["solves_per_s"] / fp64_rate, 3) if fp64_rate else None,
            "timing": "host wall clock, first submission to last completion, max over ranks",
            "per_rank": res["per_rank"]}


# ---------------------------------------------------------------------------------------------------------------------
# the reference's CPU path (oracle/_ref: the reference's own sources compiled here)
# ---------------------------------------------------------------------------------------------------------------------
def reference_cpu(size: int, steps: int, warmup: int, threads: int):
    """Warm AMGCL solves (the reference's fastest CPU pressure path, SA + SPAI0 + CG, eigen_solver=AMG) of the
    sphere-outlet workload at `size`^3 plus one projection, all host threads. Returns per-solve seconds."""
    from nereus_cfd_b200 import workloads as W
    from oracle import cpu, refcase

    case = W.sphere_outlet_3d(size, seed=2)
    types = cpu.label_cells(case.grid, case.scene)
    u, v, w = W.face_velocities(case.grid, types, case.seed)
    r = refcase.run(case, u, v, w, label_mode=1, types=types, solver=refcase.SOLVER_AMG, tol=TOL, threads=threads,
                    repeats=steps + warmup, timeout=3600)
    per = [float(t) + r.t_project for t in r.t_each[warmup:]]
    return per, r


def cpu_baseline_entry(args, scale_size):
    from oracle import refcase

    if not refcase.available():
        return None
    threads = os.cpu_count() or 1
    per, r = reference_cpu(scale_size, max(2, min(args.steps, 5)), 1, threads)
    ratio = ((scale_size + 2) ** 3) / float((args.size + 2) ** 3)
    val = ratio / statistics.mean(per)
    return {"value": round(val, 4), "unit": "solves/s", "cores": threads, "kind": "reference",
            "sample": "reference AMGCL SA+SPAI0 CG (eigen_solver=AMG) warm solve to 1e-8 + ProjectPressure of the "
                      "same sphere-outlet workload at %d^3 (%d solves, %.3f s each, %d iterations), scaled by the "
                      "cell ratio %.4f to %d^3" % (scale_size, len(per), statistics.mean(per), r.iters, ratio,
                                                   args.size)}


def run_reference(args, rank, world):
    from oracle import refcase

    if rank != 0:
        return None
    if not refcase.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/ref_harness was not built (reference sources absent)"}
    threads = os.cpu_count() or 1
    sample = args.ref_size
    per, r = reference_cpu(sample, args.steps, args.warmup, threads)
    ratio = ((sample + 2) ** 3) / float((args.size + 2) ** 3)
    lat = [t / ratio for t in per]  # seconds per full-size-equivalent solve
    total = sum(lat)
    value = args.steps / total
    desc = ("reference AMGCL SA+SPAI0 CG (eigen_solver=AMG), warm, to 1e-8, + ProjectPressure; each step one solve "
            "of the sphere-outlet workload at %d^3, scaled by the cell ratio %.4f to %d^3; %d host threads"
            % (sample, ratio, args.size, threads))
    return {"metric": METRIC, "value": round(value, 4), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": "sphere_outlet_3d_%d" % args.size, "tol": TOL, "precision": "fp64",
                       "parallelism": "host threads x%d" % threads, "sample": desc},
            "latency_ms": {"p50": round(1e3 * percentile(lat, 0.5), 3), "p99": round(1e3 * percentile(lat, 0.99), 3)},
            "cpu_baseline": {"value": round(value, 4), "unit": "solves/s", "cores": threads, "kind": "reference",
                             "sample": desc},
            "e2e": {"value": round(value, 4), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--ref-size", type=int, default=128, help="reference sample size (cells per side)")
    ap.add_argument("--fp64-steps", type=int, default=5)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--opt", action="append", default=[], help="solver option key=value (nb_options field)")
    ap.add_argument("--tanks", type=int, default=64, help="batched tanks (0: skip the batched form)")
    ap.add_argument("--tank-size", type=int, default=128)
    ap.add_argument("--slots", type=int, default=8, help="concurrent solves per device in the batched form")
    ap.add_argument("--fp64-tanks", type=int, default=4, help="tanks solved one at a time in plain FP64")
    ap.add_argument("--trace", type=int, default=200, help="requests of the serving trace (0: skip)")
    ap.add_argument("--stretched-steps", type=int, default=5, help="steps of the stretched workload (0: skip)")
    ap.add_argument("--trace-fp64", type=int, default=40, help="trace requests solved one at a time in plain FP64")
    ap.add_argument("--relabel-steps", type=int, default=10, help="timed steps of FLIP's re-labelling (0: skip)")
    ap.add_argument("--relabel-size", type=int, default=256)
    args = ap.parse_args()
    args.solver_opts = {k: int(v) if v.lstrip("-").isdigit() else float(v)
                        for k, v in (o.split("=", 1) for o in args.opt)}

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out))
        return

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = td
    # the CPU baseline runs before any GPU work, on rank 0 at N = 1 only
    cpu_base = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            cpu_base = cpu_baseline_entry(args, args.ref_size)
        except Exception as e:  # reported, never fatal to the GPU line
            cpu_base = {"unavailable": str(e)[:200]}
    out = run_b200(args, rank, world, dist)
    out["cpu_baseline"] = cpu_base
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
