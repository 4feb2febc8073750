"""The batched form (nereus_b200_batch_*) through the C ABI: many FLIP-style tanks of one grid shape advanced by the
same launches give, request by request, exactly what each one's solo solve gives.

* Every tank's pressure and corrected velocities are bit for bit those of nereus_b200_project_device on a single
  context with the same options, with the same iteration counts, for tanks with different liquid blocks (different
  unknown counts and iteration counts), a closed tank that is all liquid (singular, compatibility on), and again
  on a repeated call and on a batch that runs fewer slots than it holds.
* Each result meets its tolerance, and the autotuner recorded a launch shape for every split level.
"""
import copy

import numpy as np
import pytest

from nereus_cfd_b200 import capi, serving, workloads as W
from nereus_cfd_b200.pressure import PressureSolver

pytestmark = pytest.mark.gpu
N = 40  # 42^3 cells with the ring: levels 42, 22, 12 split, then the coarse end


def tank_jobs(count, n=N, seed=70):
    cases = [W.flip_tank_3d(n, seed=seed + 1000 * t) for t in range(count - 1)]
    jobs = [serving.job_from_case(c, tol=1e-8) for c in cases]
    # a closed tank full of liquid: no Dirichlet cell, so singular; compatibility on
    full = W.flip_tank_3d(n, seed=seed + 7, a=1.5, b=1.5)
    j = serving.job_from_case(full, tol=1e-8)
    j.needs_compat = True
    jobs.append(j)
    return jobs


def solo(job, **opts):
    import torch

    j = serving.to_device(copy.deepcopy(job))
    s = PressureSolver("mixed", **opts)
    s.InitializePressureSolver(j.grid)
    f, res = j.device_fields, capi.Result()
    capi.check(s.lib.nereus_b200_project_device(s.ctx, f["u"].data_ptr(), f["v"].data_ptr(), f["w"].data_ptr(),
                                                f["p"].data_ptr(), j.grid.rho, j.grid.dt, int(j.needs_compat), j.tol,
                                                capi.ctypes.byref(res)))
    torch.cuda.synchronize()
    s.DestroyPressureSolver()
    return serving.fetch(j), res.as_dict()


def batched(batch, jobs):
    import torch

    js = [serving.to_device(copy.deepcopy(j)) for j in jobs]
    res = batch.project(js, allow=(capi.NB_OK,))
    torch.cuda.synchronize()
    return [serving.fetch(j) for j in js], res


def assert_same(a, ra, b, rb):
    assert ra["status"] == rb["status"] == capi.NB_OK
    assert (ra["iters_inner"], ra["iters_outer"], ra["n"], ra["singular"]) == \
        (rb["iters_inner"], rb["iters_outer"], rb["n"], rb["singular"])
    assert ra["rel_res"] == rb["rel_res"] and ra["rel_res"] <= 1e-8
    for k in ("p", "u", "v", "w"):
        x, y = getattr(a.grid, k), getattr(b.grid, k)
        assert np.array_equal(x, y), (k, np.abs(x - y).max())
    assert ra["max_div"] == rb["max_div"]


@pytest.fixture(scope="module")
def jobs():
    return tank_jobs(6)


@pytest.fixture(scope="module")
def solos(jobs):
    return [solo(j) for j in jobs]


def test_batch_equals_solo_solves(nb, jobs, solos):
    with serving.Batch(len(jobs)) as b:
        for i, j in enumerate(jobs):
            b.set_layout(i, j.grid)
        out, res = batched(b, jobs)
        for (s, rs), o, r in zip(solos, out, res):
            assert_same(s, rs, o, r)
        iters = sorted(r["iters_inner"] for r in res)
        assert res[-1]["singular"] == 1
        info = b.info()
        assert info["tail_start"] >= 1 and info["loop_launches"] > 0
        for lv in info["march"]:
            assert all(v >= 1 for v in lv.values())
        # the same batch again: the captured loop and the tables are reused
        out2, res2 = batched(b, jobs)
        for (s, rs), o, r in zip(solos, out2, res2):
            assert_same(s, rs, o, r)
        # fewer requests than slots
        out3, res3 = batched(b, jobs[:3])
        for (s, rs), o, r in zip(solos[:3], out3, res3):
            assert_same(s, rs, o, r)
    assert iters[0] > 0


def test_batch_without_tuning_equals_solo(nb, jobs, solos):
    with serving.Batch(3, autotune=0) as b:
        for i, j in enumerate(jobs[3:]):
            b.set_layout(i, j.grid)
        out, res = batched(b, jobs[3:])
        for (s, rs), o, r in zip(solos[3:], out, res):
            assert_same(s, rs, o, r)
    cache = serving.tune_cache_dump()
    assert "split 42x42x42 L0 half B6" in cache


def test_batch_refuses_mixed_shapes(nb, jobs):
    other = serving.job_from_case(W.flip_tank_3d(N - 8, seed=3), tol=1e-8)
    with serving.Batch(2) as b:
        b.set_layout(0, jobs[0].grid)
        b.set_layout(1, other.grid)
        js = [serving.to_device(copy.deepcopy(jobs[0])), serving.to_device(other)]
        with pytest.raises(capi.NBError) as e:
            b.project(js)
        assert e.value.status == capi.NB_BAD_INPUT


def test_skipping_idle_tiles_changes_nothing(nb, jobs):
    """Blocks whose cells are all air or solid skip their work (skip_idle_tiles, on by default); the results are
    the ones every block working gives, bit for bit, solo and batched."""
    for j in jobs[:3]:
        a, ra = solo(j)
        b, rb = solo(j, skip_idle_tiles=0)
        assert_same(a, ra, b, rb)
    with serving.Batch(3, skip_idle_tiles=0) as b:
        for i, j in enumerate(jobs[:3]):
            b.set_layout(i, j.grid)
        out, res = batched(b, jobs[:3])
    with serving.Batch(3) as b:
        for i, j in enumerate(jobs[:3]):
            b.set_layout(i, j.grid)
        out2, res2 = batched(b, jobs[:3])
    for o, r, o2, r2 in zip(out, res, out2, res2):
        assert_same(o, r, o2, r2)
