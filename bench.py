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
    """SM clocks, power and clock-event (throttle) reasons of this process's GPU, read through NVML every 20 ms by a
    thread while the timed region runs. start() returns after the first sample, so even a timed region of a tenth of
    a second is covered; without NVML it falls back to nvidia-smi at 200 ms."""

    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("hw_power_brake_slowdown", 0x80), ("sw_power_cap", 0x4))

    def __init__(self, device: int):
        self.device = device
        self.samples = []  # (sm MHz, reasons bit mask, watts)
        self.max_mhz = None
        self.note = None
        self._stop = threading.Event()
        self._thread = None

    def _handle(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def start(self):
        try:
            nv, h = self._handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        except Exception as e:
            self.note = "NVML unavailable: %s" % str(e)[:120]
            return
        first = threading.Event()

        def run():
            while True:
                try:
                    self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                         int(nv.nvmlDeviceGetCurrentClocksEventReasons(h)),
                                         nv.nvmlDeviceGetPowerUsage(h) / 1e3))
                except Exception as e:
                    self.note = "NVML read failed: %s" % str(e)[:120]
                first.set()
                if self._stop.wait(0.02):
                    return

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        first.wait(5.0)

    def stop(self):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(5.0)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [self.note or "no samples"], "samples": 0}
        reasons = sorted({n for _, m, _ in self.samples for n, bit in self.REASONS if m & bit})
        return {"sm_mhz": statistics.median(x[0] for x in self.samples), "sm_max_mhz": self.max_mhz,
                "sm_mhz_min": min(x[0] for x in self.samples), "reasons": reasons, "samples": len(self.samples),
                "power_w_max": round(max(x[2] for x in self.samples), 1), "source": "NVML, 20 ms"}


def host_cpu():
    """The host's CPU model and logical core count (lscpu), recorded beside every CPU timing."""
    model = None
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            if line.startswith("Model name:"):
                model = line.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return {"model": model, "logical_cores": os.cpu_count()}


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
    parity = None
    if world == 1 and args.parity:
        from oracle import refcase

        if refcase.available():
            try:
                torch.cuda.synchronize()
                parity = reference_parity(args, args.ref_1e8, P.cpu().numpy(), res, mixed.IDP() >= 0)
            except Exception as e:  # reported, never fatal to the GPU line
                parity = {"unavailable": "%s: %s" % (type(e).__name__, str(e)[:300])}
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
    box2d = run_box2d(args, dev) if args.box2d_steps > 0 and world == 1 else None
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
        "parity": parity, "fp64_plain": fp64, "roofline": roof, "e2e": e2e, "clocks": clk, "gpu_launches": int(launches),
        "stretched_cylinder": stretched, "closed_box_2d": box2d, "batched_tanks": tanks, "serving_trace": trace, "flip_relabel": relabel,
    }
    return out


def run_trace(args, dev):
    """The served form (cfg5): `trace` requests of mixed dimension (3D side log-U[32, 256], 2D side log-U[64, 1024]),
    mask (closed, obstacle + outlet, free surface) and spacing (uniform, 1.04-stretched), fields drawn on the device
    just before use (a bounded number ahead, so the trace's memory stays bounded), each to 1e-8 through the server.
    A closed loop (two requests in flight per slot) gives the capacity; Poisson arrivals at each fraction of it in
    `trace_rates` give p50/p99 latency (the middle rate twice, for its run-to-run spread). The same requests one at a
    time in plain FP64 on one context (the single-solve form) are the comparison; host wall clock throughout."""
    import torch

    from nereus_cfd_b200 import capi, serving
    from nereus_cfd_b200.pressure import PressureSolver

    rng = np.random.default_rng(5)
    cases = [serving.trace_case(rng, i) for i in range(args.trace)]
    rates = [float(x) for x in args.trace_rates.split(",") if x]
    t0 = time.perf_counter()
    labels = serving.trace_labels(cases, dev)  # the requests' cell types, once, before any timing
    label_s = time.perf_counter() - t0
    out = {"requests": len(cases), "slots_per_device": args.slots, "hbm_budget_gb": 150.0,
           "mix": {"3d": sum(c.grid.dim == 3 for c in cases), "2d": sum(c.grid.dim == 2 for c in cases),
                   "stretched": sum(c.grid.nonuniform for c in cases)}}
    order = sorted(range(len(cases)), key=lambda k: -cases[k].grid.cells)[: args.slots]
    biggest = [cases[k] for k in order]
    make = lambda k: serving.device_job(cases[k], dev, TOL, labels[0][k], labels[1][k])
    with serving.Server(devices=(dev,), slots_per_device=args.slots, hbm_budget_gb=150.0, **args.solver_opts) as srv:
        # warm-up: the largest requests first, so that every slot's device arrays hold the trace's biggest shapes
        serving.serve_jobs([make(k) for k in order], srv)
        closed = serving.stream_serve(srv, cases, dev, TOL, rate=None, inflight=2 * args.slots, labels=labels)
        cap = closed["solves_per_s"]
        out["closed_loop"] = closed
        out["poisson"] = [serving.stream_serve(srv, cases, dev, TOL, rate=f * cap, seed=11 + k, labels=labels)
                          for k, f in enumerate(rates)]
        if rates:
            m = len(rates) // 2
            again = serving.stream_serve(srv, cases, dev, TOL, rate=rates[m] * cap, seed=11 + m, labels=labels)
            first = out["poisson"][m]
            out["poisson_repeat"] = again
            out["repeat_spread"] = {q: round(abs(again[q] - first[q]) / max(first[q], 1e-9), 3)
                                    for q in ("p50_ms", "p99_ms")}
    # one at a time in plain FP64 on one context, the same requests made the same way, warmed on the largest
    s = PressureSolver("fp64", device=dev, **args.solver_opts)
    lib = capi.load()

    def one(j):
        s.EnsureSystem(j.grid)
        f, res = j.device_fields, capi.Result()
        capi.check(lib.nereus_b200_project_device(s.ctx, f["u"].data_ptr(), f["v"].data_ptr(), f["w"].data_ptr(),
                                                  f["p"].data_ptr(), j.grid.rho, j.grid.dt, int(j.needs_compat), TOL,
                                                  ctypes.byref(res)), allow=(0, 1))
        torch.cuda.synchronize()
        j.device_fields = None

    warm = make(order[0])
    s.InitializePressureSolver(warm.grid)
    one(warm)
    stream = serving.JobStream(cases, dev, TOL, labels=labels)
    t0 = time.perf_counter()
    for j in stream:
        one(j)
    fp64_sec = time.perf_counter() - t0
    s.DestroyPressureSolver()
    fp64_rate = len(cases) / fp64_sec
    out["fp64_one_at_a_time"] = {"value": round(fp64_rate, 3), "unit": "solves/s", "requests": len(cases),
                                 "seconds": round(fp64_sec, 3), "make_seconds": round(stream.make_seconds, 3)}
    out["speedup_over_fp64_one_at_a_time"] = round(cap / fp64_rate, 3)
    out["timing"] = ("host wall clock; latency from submission to completion (and from the arrival time under "
                     "Poisson arrivals); cell types labelled once before timing (%.1f s), velocities drawn on the "
                     "device by a producer thread a bounded number of requests ahead" % label_s)
    return out


def run_case_leg(args, dev, case, tol, compat, steps, name):
    """One workload solved again and again, mixed and plain FP64, fields device-resident and restored from a copy
    each step (inside the timed step), CUDA events around each step after three warm-up steps."""
    import torch

    from nereus_cfd_b200 import capi
    from nereus_cfd_b200.pressure import MACGrid, PressureSolver

    lib = capi.load()
    types = capi.label_cells(case.grid, case.scene)
    from nereus_cfd_b200 import workloads as W

    u, v, w = W.face_velocities(case.grid, types, case.seed, case.velocity_rule, case.fp32_velocity)
    td = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to("cuda")
    wz = w if case.grid.dim == 3 else np.zeros(1)
    orig = [td(u), td(v), td(wz), torch.zeros(case.grid.cells, dtype=torch.float64, device="cuda")]
    work = [t.clone() for t in orig]
    out = {"workload": name, "unknowns": None, "tol": tol}
    for prec in ("mixed", "fp64"):
        s = PressureSolver(prec, device=dev, **args.solver_opts)
        s.InitializePressureSolver(MACGrid.from_case(case, types, u, v, wz))
        res = capi.Result()
        evs = []
        for k in range(3 + steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for x, y in zip(work, orig):
                x.copy_(y)
            capi.check(lib.nereus_b200_project_device(s.ctx, *[t.data_ptr() for t in work], case.rho, case.dt,
                                                      int(compat), tol, ctypes.byref(res)), allow=(0, 1))
            b.record()
            if k >= 3:
                evs.append((a, b))
        torch.cuda.synchronize()
        ms = [a.elapsed_time(b) for a, b in evs]
        out[prec] = {"value": round(1e3 / statistics.mean(ms), 3), "unit": "solves/s",
                     "p50_ms": round(percentile(ms, 0.5), 3), "iters_inner": res.iters_inner,
                     "iters_outer": res.iters_outer, "rel_res": res.rel_res, "max_div": res.max_div,
                     "status": res.status, "steps": len(ms)}
        out["unknowns"] = res.n
        s.DestroyPressureSolver()
    out["speedup_mixed_over_fp64"] = round(out["mixed"]["value"] / out["fp64"]["value"], 3)
    return out


def run_stretched(args, dev):
    """The stretched workload (cfg3): 192x128x128 on [0,2.2]x[0,0.41]^2, widths x 1.04 per cell away from a 24-cell
    band at x = 0.5, a solid cylinder along z, inflow at x = 0, p = 0 outlet at x = 2.2, seeded N(0,1) faces; mixed
    and plain FP64 to 1e-8."""
    from nereus_cfd_b200 import workloads as W

    return run_case_leg(args, dev, W.stretched_cylinder_3d(192, 128, 128, seed=3), TOL, False, args.stretched_steps,
                        "stretched_cylinder_192x128x128")


def run_box2d(args, dev):
    """The 2D closed box (cfg1): 128^2 uniform on the unit square, all fluid, no-slip walls (all-Neumann, the
    compatibility condition on), seeded N(0,1) faces; mixed and plain FP64 to 1e-10."""
    from nereus_cfd_b200 import workloads as W

    return run_case_leg(args, dev, W.closed_box_2d(128, seed=1), 1e-10, True, args.box2d_steps, "closed_box_2d_128")


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
    """The batched form (cfg4): `tanks` FLIP-style n^3 tanks (liquid where x < a, z < b; a, b ~ U(0.3, 0.7) per tank),
    each step one pressure projection of every tank to 1e-8 as ONE batched call (nereus_b200_batch_project_device:
    every kernel of a CG iteration is one launch over all tanks still iterating, the iteration a captured graph with
    a WHILE node, launch shapes autotuned on the first call). The tanks' fields stay on the device and are restored
    from a copy inside every step. Against the same tanks one at a time, each on its own context holding its layout,
    in plain FP64 (the single-solve form) and in the mixed form. CUDA events on one stream; steps repeated until the
    timed region passes one second. With N ranks the tanks are split by the least-loaded plan; max over ranks."""
    import torch

    from nereus_cfd_b200 import capi, serving
    from nereus_cfd_b200.pressure import PressureSolver

    lib = capi.load()
    cases = serving.tank_batch(args.tanks, args.tank_size)
    stream = torch.cuda.current_stream()
    summary = {}

    def execute(mine):
        jobs = [serving.to_device(serving.job_from_case(c, tol=TOL), dev) for c in mine]
        if not jobs:
            return {"seconds": 0.0, "completed": 0, "latencies": []}
        keys = ("u", "v", "w", "p")
        # every tank's field k is a slice of one buffer, so a step restores all tanks with one copy per field
        big, orig_big = {}, {}
        for k in keys:
            n = jobs[0].device_fields[k].numel()
            big[k] = torch.empty(n * len(jobs), dtype=torch.float64, device="cuda")
            for i, j in enumerate(jobs):
                big[k][i * n:(i + 1) * n].copy_(j.device_fields[k])
                j.device_fields[k] = big[k][i * n:(i + 1) * n]
            orig_big[k] = big[k].clone()
        orig = [{k: orig_big[k][i * big[k].numel() // len(jobs):(i + 1) * big[k].numel() // len(jobs)]
                 for k in keys} for i in range(len(jobs))]

        def restore(i):
            for k in keys:
                jobs[i].device_fields[k].copy_(orig[i][k])

        def restore_all():
            for k in keys:
                big[k].copy_(orig_big[k])

        def events():
            return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        # ---- the batched form ----
        batch = serving.Batch(len(jobs), device=dev, stream=stream.cuda_stream, **args.solver_opts)
        for i, j in enumerate(jobs):
            batch.set_layout(i, j.grid)
        items = batch.items(jobs)

        def step():
            restore_all()
            return batch.project(jobs, items=items)

        for _ in range(2):  # the first call tunes and captures
            step()
        a, b = events()
        a.record(stream)
        step()
        b.record(stream)
        torch.cuda.synchronize()
        one = a.elapsed_time(b) / 1e3
        steps = max(args.tank_steps, int(1.0 / max(one, 1e-6)) + 1)
        lat = []
        l0 = lib.nereus_b200_kernel_launches()
        a, b = events()
        a.record(stream)
        for _ in range(steps):
            x, y = events()
            x.record(stream)
            res = step()
            y.record(stream)
            lat.append((x, y))
        b.record(stream)
        torch.cuda.synchronize()
        secs = a.elapsed_time(b) / 1e3
        launches = lib.nereus_b200_kernel_launches() - l0
        lat = [x.elapsed_time(y) for x, y in lat]
        info = batch.info()
        batch.close()
        out = {"seconds": secs, "completed": steps * len(jobs), "steps": steps, "latencies": lat,
               "iters_inner": [r["iters_inner"] for r in res], "rel_res_max": max(r["rel_res"] for r in res),
               "status": sorted({r["status"] for r in res}), "gpu_launches": launches, "batch": info}

        # ---- one at a time, each tank on its own context (its layout kept), fields restored each time ----
        def one_at_a_time(precision):
            ss = []
            for j in jobs:
                s = PressureSolver(precision, device=dev, stream=stream.cuda_stream, **args.solver_opts)
                s.InitializePressureSolver(j.grid)
                ss.append(s)
            r = capi.Result()

            def solve(i):
                restore(i)
                f = jobs[i].device_fields
                capi.check(lib.nereus_b200_project_device(ss[i].ctx, f["u"].data_ptr(), f["v"].data_ptr(),
                                                          f["w"].data_ptr(), f["p"].data_ptr(), jobs[i].grid.rho,
                                                          jobs[i].grid.dt, 0, TOL, ctypes.byref(r)),
                           allow=(0, 1))

            for i in range(len(jobs)):  # warm: each context's graphs (captured on a layout's second solve)
                solve(i)
                solve(i)
            a, b = events()
            a.record(stream)
            for i in range(len(jobs)):
                solve(i)
            b.record(stream)
            torch.cuda.synchronize()
            sec = a.elapsed_time(b) / 1e3
            for s in ss:
                s.DestroyPressureSolver()
            return {"value": round(len(jobs) / sec, 3), "unit": "solves/s", "tanks": len(jobs),
                    "seconds": round(sec, 4)}

        out["fp64_one_at_a_time"] = one_at_a_time("fp64")
        out["mixed_one_at_a_time"] = one_at_a_time("mixed")
        summary.update(out)
        return out

    res = serving.run_sharded(cases, lambda c: c.grid.cells, execute, dist)
    fp64 = summary.get("fp64_one_at_a_time", {}).get("seconds")
    mixed1 = summary.get("mixed_one_at_a_time", {}).get("seconds")
    if dist:
        vals = [None] * world
        dist.all_gather_object(vals, (fp64, mixed1))
        fp64 = max(v[0] for v in vals if v[0] is not None)
        mixed1 = max(v[1] for v in vals if v[1] is not None)
    fp64_rate = args.tanks / fp64 if fp64 else None
    mixed1_rate = args.tanks / mixed1 if mixed1 else None
    its = summary.get("iters_inner", [])
    lat = summary.get("latencies", [])
    return {"workload": "flip_tanks_%dx%d^3" % (args.tanks, args.tank_size), "tanks": args.tanks,
            "form": "one batched call per step (nereus_b200_batch_project_device)",
            "value": round(res["solves_per_s"], 3), "unit": "solves/s", "steps": summary.get("steps"),
            "seconds": round(res["seconds"], 4), "step_p50_ms": round(percentile(lat, 0.5), 3) if lat else None,
            "step_p99_ms": round(percentile(lat, 0.99), 3) if lat else None, "scaling": "strong",
            "iters_inner_rank0": [int(min(its)), int(max(its))] if its else None,
            "rel_res_max_rank0": summary.get("rel_res_max"), "status_rank0": summary.get("status"),
            "gpu_launches_rank0": summary.get("gpu_launches"), "batch_rank0": summary.get("batch"),
            "fp64_one_at_a_time": {"value": round(fp64_rate, 3) if fp64_rate else None, "unit": "solves/s",
                                   "tanks": args.tanks},
            "mixed_one_at_a_time": {"value": round(mixed1_rate, 3) if mixed1_rate else None, "unit": "solves/s",
                                    "tanks": args.tanks},
            "speedup_over_fp64_one_at_a_time": round(res["solves_per_s"] / fp64_rate, 3) if fp64_rate else None,
            "speedup_over_mixed_one_at_a_time": round(res["solves_per_s"] / mixed1_rate, 3) if mixed1_rate else None,
            "timing": "CUDA events on one stream, fields restored inside each step; max over ranks",
            "per_rank": res["per_rank"]}


# ---------------------------------------------------------------------------------------------------------------------
# the reference's CPU path (oracle/_ref: the reference's own sources compiled here), at the bench's own size
# ---------------------------------------------------------------------------------------------------------------------
def reference_solve(size: int, solver: int, tol: float, repeats: int, threads: int):
    """The reference's SolvePressure + ProjectPressure on the sphere-outlet workload at `size`^3 (rank 0's seed, the
    same fields the B200 arm projects), labels from the oracle (bit-exact with the reference's own), all `threads`
    host threads. One cold solve (assembly and, for AMGCL, its hierarchy), then `repeats` warm solves of the same
    system; the result leaves out the matrix (lean)."""
    from nereus_cfd_b200 import workloads as W
    from oracle import cpu, refcase

    case = W.sphere_outlet_3d(size, seed=2)
    types = cpu.label_cells(case.grid, case.scene)
    u, v, w = W.face_velocities(case.grid, types, case.seed)
    return refcase.run(case, u, v, w, label_mode=1, types=types, solver=solver, tol=tol, threads=threads,
                       repeats=repeats, timeout=3600, lean=True)


def cpu_baseline_entry(args):
    """The reference's AMGCL path (SA + SPAI0 + CG, eigen_solver=AMG, its fastest CPU path) on the bench's own
    workload at full size: one cold solve, then one warm solve + ProjectPressure timed (about 10-30 s of CPU work).
    Returns the cpu_baseline record and the run (its max |div u| at 1e-8 is the divergence reference)."""
    from oracle import refcase

    if not refcase.available():
        return None, None
    threads = os.cpu_count() or 1
    r = reference_solve(args.size, refcase.SOLVER_AMG, TOL, 1, threads)
    per = float(r.t_each[0]) + r.t_project
    return ({"value": round(1.0 / per, 4), "unit": "solves/s", "cores": threads, "kind": "reference",
             "host": host_cpu(),
             "sample": "reference AMGCL SA+SPAI0 CG (eigen_solver=AMG) on sphere_outlet_3d_%d itself (no scaling): "
                       "one cold solve (%.2f s with AMG setup), then one warm solve to 1e-8 (%.3f s, %d iterations) "
                       "+ ProjectPressure (%.3f s); the warm solve + projection is the value"
                       % (args.size, r.t_solve_cold, float(r.t_each[0]), r.iters, r.t_project)}, r)


def reference_parity(args, ref_1e8, P, res, idp_mask):
    """north_star (1) on the headline solve: the B200 pressure (1e-8) against the reference's own solve of the same
    system at 1e-12 (AMGCL; its Eigen CG needs thousands of iterations at this size), as relative L2 over the
    unknowns (mean-free when singular), and the B200 max |div u| over the reference's at the same 1e-8."""
    from oracle import refcase

    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    r12 = reference_solve(args.size, refcase.SOLVER_AMG, 1e-12, 0, threads)
    x_ref = r12.p[idp_mask]
    x = P[idp_mask]
    if r12.singular:
        x, x_ref = x - x.mean(), x_ref - x_ref.mean()
    err = float(np.linalg.norm(x - x_ref) / max(np.linalg.norm(x_ref), 1e-300))
    out = {"reference": "AMGCL SA+SPAI0 CG (eigen_solver=AMG) to 1e-12, %d iterations, rel_res %.2e"
                        % (r12.iters, r12.rel_res),
           "pressure_rel_l2": err, "pressure_bar": 1e-6, "rel_res": res.rel_res,
           "max_div": res.max_div, "seconds": round(time.perf_counter() - t0, 2)}
    if ref_1e8 is not None:
        out["max_div_ref_1e8"] = ref_1e8.max_div
        out["max_div_ratio"] = res.max_div / max(ref_1e8.max_div, 1e-300)
        out["max_div_bar"] = 10.0
        if ref_1e8.p is not None and ref_1e8.p.size == r12.p.size:
            # for context: the reference's own solve at the same 1e-8 against its 1e-12 solve
            x8 = ref_1e8.p[idp_mask]
            x12 = r12.p[idp_mask]
            if r12.singular:
                x8, x12 = x8 - x8.mean(), x12 - x12.mean()
            out["reference_1e8_pressure_rel_l2"] = float(np.linalg.norm(x8 - x12) / max(np.linalg.norm(x12), 1e-300))
            out["reference_1e8_rel_res"] = ref_1e8.rel_res
    out["ok"] = bool(err <= 1e-6 and res.rel_res <= TOL and out.get("max_div_ratio", 0.0) <= 10.0)
    return out


def run_reference(args, rank, world):
    from oracle import refcase

    if rank != 0:
        return None
    if not refcase.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/ref_harness was not built (reference sources absent)"}
    threads = os.cpu_count() or 1
    r = reference_solve(args.size, refcase.SOLVER_AMG, TOL, args.warmup + args.steps, threads)
    lat = [float(t) + r.t_project for t in r.t_each[args.warmup:]]
    total = sum(lat)
    value = args.steps / total
    host = host_cpu()
    desc = ("reference AMGCL SA+SPAI0 CG (eigen_solver=AMG), warm solves to 1e-8 of sphere_outlet_3d_%d itself (%d "
            "iterations) + ProjectPressure, one solve per step after one cold solve (%.2f s with AMG setup) and %d "
            "warm-up solves; %d host threads" % (args.size, r.iters, r.t_solve_cold, args.warmup, threads))
    out = {"metric": METRIC, "value": round(value, 4), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
           "config": {"workload": "sphere_outlet_3d_%d" % args.size, "tol": TOL, "precision": "fp64",
                      "parallelism": "host threads x%d" % threads, "sample": desc, "host": host},
           "latency_ms": {"p50": round(1e3 * percentile(lat, 0.5), 3), "p99": round(1e3 * percentile(lat, 0.99), 3)},
           "solve": {"iters": r.iters, "rel_res": r.rel_res, "max_div": r.max_div},
           "cpu_baseline": {"value": round(value, 4), "unit": "solves/s", "cores": threads, "kind": "reference",
                            "sample": desc},
           "e2e": {"value": round(value, 4), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.eigen_cg:
        # the reference's Eigen CG + diagonal preconditioner (its default CPU solver and the parity oracle's), one
        # solve of the same system to 1e-8; slow at this size, so one step only
        e = reference_solve(args.size, refcase.SOLVER_CG, TOL, 0, threads)
        sec = e.t_solve_cold + e.t_project
        out["eigen_cg"] = {"value": round(1.0 / sec, 5), "unit": "solves/s", "steps": 1, "seconds": round(sec, 3),
                           "iters": e.iters, "rel_res": e.rel_res, "max_div": e.max_div,
                           "sample": "Eigen ConjugateGradient + DiagonalPreconditioner (eigen_solver=CG), one cold "
                                     "solve to 1e-8 of sphere_outlet_3d_%d + ProjectPressure, %d host threads"
                                     % (args.size, threads)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--no-eigen-cg", dest="eigen_cg", action="store_false",
                    help="reference arm: skip the one Eigen-CG solve")
    ap.add_argument("--no-parity", dest="parity", action="store_false",
                    help="skip the comparison with the reference's own solve at 1e-12")
    ap.add_argument("--fp64-steps", type=int, default=5)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--opt", action="append", default=[], help="solver option key=value (nb_options field)")
    ap.add_argument("--tanks", type=int, default=64, help="batched tanks (0: skip the batched form)")
    ap.add_argument("--tank-size", type=int, default=128)
    ap.add_argument("--slots", type=int, default=4, help="concurrent solves per device of the serving trace")
    ap.add_argument("--tank-steps", type=int, default=5, help="batched steps at least (the timed region >= 1 s)")
    ap.add_argument("--trace", type=int, default=2000, help="requests of the serving trace (0: skip)")
    ap.add_argument("--trace-rates", default="0.2,0.4,0.6,0.8,1.0",
                    help="Poisson arrival rates of the trace as fractions of the closed-loop capacity")
    ap.add_argument("--stretched-steps", type=int, default=5, help="steps of the stretched workload (0: skip)")
    ap.add_argument("--box2d-steps", type=int, default=10, help="steps of the 2D 128^2 closed box (0: skip)")
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
    cpu_base, ref_1e8 = None, None
    if world == 1 and not args.no_cpu_baseline:
        try:
            cpu_base, ref_1e8 = cpu_baseline_entry(args)
        except Exception as e:  # reported, never fatal to the GPU line
            cpu_base = {"unavailable": str(e)[:200]}
    args.ref_1e8 = ref_1e8
    out = run_b200(args, rank, world, dist)
    out["cpu_baseline"] = cpu_base
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
