"""The server on the B200 (nereus_b200_server_* through nereus_cfd_b200.serving): a mix of different requests run
concurrently (several slots on one device) gives each request exactly what it gives alone through
nereus_b200_project / _ex; admission by the memory budget; the statistics."""
import numpy as np
import pytest

from conftest import load_golden, scheme_golden_names
from nereus_cfd_b200 import capi, serving
from nereus_cfd_b200 import workloads as W
from nereus_cfd_b200.pressure import MACGrid, PressureSolver

pytestmark = pytest.mark.gpu


def mix():
    cases = [W.sphere_outlet_3d(24, seed=40), W.flip_tank_3d(20, seed=41), W.flip_tank_3d(20, seed=42),
             W.closed_box_2d(48, seed=43), W.stretched_cylinder_3d(24, 16, 16, seed=44),
             W.sphere_outlet_3d(16, seed=45), W.pressure_outlet_3d(14, seed=46), W.flip_tank_3d(32, seed=47)]
    jobs = [serving.job_from_case(c, tol=1e-9) for c in cases]
    # one incremental request from its fixture
    name = [n for n in scheme_golden_names() if n.startswith("incremental_")][0]
    case, meta, z = load_golden(name)
    m = MACGrid(case.grid, z["types"].copy(), z["u"].copy(), z["v"].copy(), z["w"].copy(), z["p_in"].copy(),
                meta["rho"], meta["dt"])
    jobs.append(serving.Job(m, tol=1e-9, needs_compat=meta["needs_compat"], scheme=capi.SCHEME_INCREMENTAL,
                            p_prev=z["p_prev"].copy()))
    return jobs


def alone(job, precision):
    m = job.grid
    s = PressureSolver(precision)
    s.InitializePressureSolver(m, job.scheme)
    ant = None
    if job.p_prev is not None:
        ant = MACGrid(m.grid, m.types, m.u, m.v, m.w, job.p_prev, m.rho, m.dt)
    r = s.SolvePressure(m, tol=job.tol, needs_compat=job.needs_compat, grid_ant=ant)
    s.DestroyPressureSolver()
    return r


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_mix_equals_alone(nb, precision):
    served = mix()
    ref = mix()
    with serving.Server(slots_per_device=4, precision=precision) as srv:
        st = serving.serve(served, srv)
    assert st["completed"] == len(served) and st["failed"] == 0
    assert st["p50_ms"] <= st["p99_ms"] and st["solves_per_s"] > 0
    for a, b in zip(served, ref):
        r = alone(b, precision)
        assert a.status == capi.NB_OK and r.status == capi.NB_OK
        assert a.result["iters_inner"] == r.iters_inner
        for f in ("p", "u", "v", "w"):
            assert np.array_equal(getattr(a.grid, f), getattr(b.grid, f)), f


def test_device_fields_equal_host_fields(nb):
    host = mix()
    dev = [serving.to_device(j) for j in mix()]
    with serving.Server(slots_per_device=4) as srv:
        serving.serve(host, srv)
    with serving.Server(slots_per_device=4) as srv:
        serving.serve(dev, srv)
    for a, b in zip(host, dev):
        serving.fetch(b)
        assert a.status == b.status == capi.NB_OK
        assert a.result["iters_inner"] == b.result["iters_inner"]
        for f in ("p", "u", "v", "w"):
            assert np.array_equal(getattr(a.grid, f), getattr(b.grid, f)), f


def test_admission_budget(nb):
    job = mix()[0]
    with serving.Server(hbm_budget_gb=0.01) as srv:
        with pytest.raises(capi.NBError) as e:
            srv.submit(job)
        assert e.value.status == capi.NB_BAD_INPUT
    need = serving.request_bytes(job) / 1e9
    # a budget for one request at a time: all still complete, one after another
    jobs = mix()[:4]
    with serving.Server(hbm_budget_gb=max(serving.request_bytes(j) for j in jobs) / 1e9 * 1.01,
                        slots_per_device=4) as srv:
        st = serving.serve(jobs, srv)
    assert need > 0 and st["completed"] == 4


def test_poll_and_bad_requests(nb):
    job = mix()[0]
    with serving.Server() as srv:
        t = srv.submit(job)
        st = srv.poll(t)
        assert st in (capi.NB_BUSY, capi.NB_OK)
        assert srv.wait(t, 60.0) == capi.NB_OK
        assert srv.poll(t) == capi.NB_OK
        res = capi.Result()
        assert srv.lib.nereus_b200_poll(srv.srv, 987654321, None) == capi.NB_BAD_INPUT
        bad = serving.Job(job.grid, scheme=capi.SCHEME_INCREMENTAL)  # no previous pressure
        with pytest.raises(capi.NBError):
            srv.submit(bad)
