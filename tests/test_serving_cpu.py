"""Host logic of the batch/serving layer without a GPU: the least-loaded plan, the request cost, the server's
refusal to start without a device, and the sharded run over two gloo ranks (the oracle solves each rank's share)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT, cuda_ok
from nereus_cfd_b200 import build, capi, serving
from nereus_cfd_b200 import workloads as W


@pytest.fixture(scope="module", autouse=True)
def lib():
    build.build()
    return capi.load()


def test_plan_is_least_loaded_in_order():
    assert serving.plan([5, 3, 3, 1, 4], 2) == [0, 1, 1, 0, 0]
    assert serving.plan([1, 1, 1, 1], 3) == [0, 1, 2, 0]  # ties go to the lowest index
    assert serving.plan([], 4) == []
    costs = np.random.default_rng(3).uniform(1, 100, 200)
    owner = serving.plan(costs, 4)
    loads = [costs[np.array(owner) == d].sum() for d in range(4)]
    assert max(loads) - min(loads) <= costs.max()


def test_plan_rejects_bad_arguments(lib):
    out = (serving.ctypes.c_int * 1)()
    c = np.ones(1)
    assert lib.nereus_b200_plan(capi.ptr(c), 1, 0, out) == capi.NB_BAD_INPUT


def test_request_bytes_grow_with_the_grid(lib):
    small = lib.nereus_b200_request_bytes(3, 34, 34, 34, capi.PRECISION_MIXED)
    big = lib.nereus_b200_request_bytes(3, 258, 258, 258, capi.PRECISION_MIXED)
    fp64 = lib.nereus_b200_request_bytes(3, 258, 258, 258, capi.PRECISION_FP64)
    assert 0 < small < big < fp64
    assert big < 150e9 / 8  # eight 256^3 solves fit one device's default budget


@pytest.mark.skipif(cuda_ok(), reason="checks the no-GPU behaviour")
def test_server_needs_a_device():
    with pytest.raises(capi.NBError) as e:
        serving.Server()
    assert e.value.status == capi.NB_NO_DEVICE


# ---- two gloo ranks ----
def _jobs():
    from oracle import cpu

    cases = [W.sphere_outlet_3d(8, seed=30), W.flip_tank_3d(8, seed=31), W.closed_box_2d(12, seed=32),
             W.sphere_outlet_3d(10, seed=33), W.flip_tank_3d(10, seed=34), W.pressure_outlet_3d(8, seed=35)]
    jobs = []
    for c in cases:
        types = cpu.label_cells(c.grid, c.scene)
        jobs.append(serving.job_from_case(c, tol=1e-10, types=types))
    return jobs


def _oracle_execute(jobs):
    """Each job solved by the oracle (test infrastructure), standing in for a rank's device."""
    import time

    from oracle import cpu

    t0 = time.perf_counter()
    for j in jobs:
        m = j.grid
        t1 = time.perf_counter()
        r = cpu.solve_projection(m.grid, m.types, m.u, m.v, m.w, m.p, m.rho, m.dt, j.needs_compat, j.tol)
        m.p[:], m.u[:], m.v[:] = r.p, r.u, r.v
        if m.w.size:
            m.w[:] = r.w
        j.status, j.latency_ms, j.result = 0, 1e3 * (time.perf_counter() - t1), {"rel_res": r.rel_res}
    return {"seconds": time.perf_counter() - t0, "completed": len(jobs), "latencies": [j.latency_ms for j in jobs]}


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        jobs = _jobs()
        summary = serving.run_sharded(jobs, lambda j: j.cells, _oracle_execute, dist)
        owner = serving.plan([j.cells for j in jobs], world)
        mine = [i for i, o in enumerate(owner) if o == rank]
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), mine=np.array(mine, dtype=np.int64),
                 p=np.concatenate([jobs[i].grid.p for i in mine]) if mine else np.zeros(0),
                 completed=summary["completed"], world=summary["world"], seconds=summary["seconds"],
                 rank_seconds=np.array([r["seconds"] for r in summary["per_rank"]]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_run_over_two_gloo_ranks(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    outs = [np.load(os.path.join(tmp_path, "rank%d.npz" % r)) for r in range(world)]
    mine = [set(o["mine"].tolist()) for o in outs]
    assert mine[0].isdisjoint(mine[1]) and (mine[0] | mine[1]) == set(range(6))  # every job once
    for o in outs:
        assert int(o["completed"]) == 6 and int(o["world"]) == 2
        assert float(o["seconds"]) == float(o["rank_seconds"].max())  # max over ranks
    # each rank's results equal the same jobs solved in one process
    ref = _jobs()
    _oracle_execute(ref)
    for o in outs:
        expect = np.concatenate([ref[i].grid.p for i in o["mine"]]) if len(o["mine"]) else np.zeros(0)
        assert np.array_equal(o["p"], expect)
