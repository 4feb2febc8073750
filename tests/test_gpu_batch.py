"""The batched form (nereus_b200_batch_*) through the C ABI: many FLIP-style tanks of one grid shape advanced by the
same launches.

* A request's result does not depend on what else runs beside it: alone in a batch, in a mix of six tanks, in
  another slot order, with or without the autotuner's launch shapes, its pressure and corrected velocities are the
  same bit for bit.
* Against a single context's solve of the same request (nereus_b200_project_device, same options) the batched
  kernels round in FP32 where the compiler fused products differently, so they agree within the stated tolerance:
  both reach rel_res <= 1e-8, the mean-free pressures within 1e-6 relative L2, the velocities within 1e-6 relative
  L2, max |div u| within 10x, the iteration counts within one.
* The tanks differ in their liquid blocks (unknown and iteration counts); one is all liquid (singular, the
  compatibility condition on); repeated calls and a batch running fewer slots than it holds are covered.
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
    """bit for bit"""
    assert ra["status"] == rb["status"] == capi.NB_OK
    assert (ra["iters_inner"], ra["iters_outer"], ra["n"], ra["singular"]) == \
        (rb["iters_inner"], rb["iters_outer"], rb["n"], rb["singular"])
    assert ra["rel_res"] == rb["rel_res"] and ra["rel_res"] <= 1e-8
    for k in ("p", "u", "v", "w"):
        x, y = getattr(a.grid, k), getattr(b.grid, k)
        assert np.array_equal(x, y), (k, np.abs(x - y).max())
    assert ra["max_div"] == rb["max_div"]


def rel(x, y):
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


def assert_close(a, ra, b, rb):
    """within the stated tolerance: b is the single-context solve"""
    assert ra["status"] == rb["status"] == capi.NB_OK
    assert (ra["n"], ra["singular"], ra["iters_outer"]) == (rb["n"], rb["singular"], rb["iters_outer"])
    assert abs(ra["iters_inner"] - rb["iters_inner"]) <= 1
    assert ra["rel_res"] <= 1e-8 and rb["rel_res"] <= 1e-8
    pa, pb = a.grid.p, b.grid.p
    if ra["singular"]:
        mask = a.grid.types == W.FLUID
        pa, pb = pa[mask] - pa[mask].mean(), pb[mask] - pb[mask].mean()
    assert rel(pa, pb) <= 1e-6
    for k in ("u", "v", "w"):
        assert rel(getattr(a.grid, k), getattr(b.grid, k)) <= 1e-6, k
    assert ra["max_div"] <= 10.0 * rb["max_div"] + 1e-12


@pytest.fixture(scope="module")
def jobs():
    return tank_jobs(6)


@pytest.fixture(scope="module")
def solos(jobs):
    return [solo(j) for j in jobs]


def test_batch_matches_solo_within_tolerance(nb, jobs, solos):
    with serving.Batch(len(jobs)) as b:
        for i, j in enumerate(jobs):
            b.set_layout(i, j.grid)
        out, res = batched(b, jobs)
        for (s, rs), o, r in zip(solos, out, res):
            assert_close(o, r, s, rs)
        assert res[-1]["singular"] == 1
        info = b.info()
        assert info["tail_start"] >= 1 and info["loop_launches"] > 0
        for lv in info["march"]:
            assert all(v >= 1 for v in lv.values())
        # the same batch again: the captured loop and the tables are reused, the bits repeat
        out2, res2 = batched(b, jobs)
        for o, r, o2, r2 in zip(out, res, out2, res2):
            assert_same(o2, r2, o, r)
        # fewer requests than slots
        out3, res3 = batched(b, jobs[:3])
        for o, r, o3, r3 in zip(out, res, out3, res3):
            assert_same(o3, r3, o, r)


def test_alone_equals_in_the_mix(nb, jobs):
    with serving.Batch(len(jobs)) as b:
        for i, j in enumerate(jobs):
            b.set_layout(i, j.grid)
        mix, rmix = batched(b, jobs)
    rev = list(reversed(jobs))
    with serving.Batch(len(jobs)) as b:
        for i, j in enumerate(rev):
            b.set_layout(i, j.grid)
        back, rback = batched(b, rev)
    for o, r, o2, r2 in zip(mix, rmix, reversed(back), reversed(rback)):
        assert_same(o2, r2, o, r)
    for k in (0, 2, 5):
        with serving.Batch(1) as b:
            b.set_layout(0, jobs[k].grid)
            alone, ralone = batched(b, [jobs[k]])
        assert_same(alone[0], ralone[0], mix[k], rmix[k])


def test_batch_without_tuning_equals_tuned(nb, jobs):
    with serving.Batch(3) as b:
        for i, j in enumerate(jobs[3:]):
            b.set_layout(i, j.grid)
        tuned, rt = batched(b, jobs[3:])
    with serving.Batch(3, autotune=0) as b:
        for i, j in enumerate(jobs[3:]):
            b.set_layout(i, j.grid)
        plain, rp = batched(b, jobs[3:])
    for o, r, o2, r2 in zip(tuned, rt, plain, rp):
        assert_same(o2, r2, o, r)
    cache = serving.tune_cache_dump()
    assert "split 42x42x42 L0 half B3" in cache


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
