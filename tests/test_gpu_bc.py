"""The boundary-condition replay on the B200 (nereus_b200_bc_*) against the reference's own EnforceVelocityBC and
EnforcePressureBC (tests/golden/bc_*.npz: the lists its MAC::BuildBoundaryLists made, the values its boundary
functions gave, and the fields before and after): bit for bit, ApplyOutflowFlux included; without boundary
functions against the oracle's replay; and replayed from a CUDA graph."""
import numpy as np
import pytest

from conftest import bc_golden_names, load_golden
from nereus_cfd_b200.boundary import BoundaryReplay
from oracle import cpu

pytestmark = pytest.mark.gpu
NAMES = bc_golden_names()


def _setup(name):
    import torch

    case, meta, z = load_golden(name)
    g = case.grid
    nz = g.Nz if g.dim == 3 else 1
    bc = BoundaryReplay(dict(z), g.dim, g.Nx, g.Ny, nz)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to("cuda")
    fields = [d(z["u_in"]), d(z["v_in"]), d(z["w_in"]) if g.dim == 3 else None, d(z["p_in"])]
    return case, z, bc, fields, d


def _host(fields):
    return [f.cpu().numpy() if f is not None else np.zeros(0) for f in fields]


@pytest.mark.parametrize("name", NAMES)
def test_replay_matches_reference(nb, name):
    import torch

    case, z, bc, (u, v, w, p), d = _setup(name)
    bc.EnforceVelocityBC(u, v, w, d(z["presc_value"]) if len(z["presc_value"]) else None)
    bc.EnforcePressureBC(p, d(z["ring_value"]) if len(z["ring_value"]) else None)
    torch.cuda.synchronize()
    hu, hv, hw, hp = _host([u, v, w, p])
    assert np.array_equal(hu, z["u_out"])
    assert np.array_equal(hv, z["v_out"])
    assert np.array_equal(hw, z["w_out"])
    assert np.array_equal(hp, z["p_out"])
    lv, lp = bc.levels()
    assert 1 <= lv <= 16 and 1 <= lp <= 16
    bc.close()


@pytest.mark.parametrize("name", NAMES)
def test_replay_without_boundary_functions_matches_oracle(nb, name):
    """No boundary velocity function: the prescribed entries stay unwritten; no pressure function: 0 there."""
    import torch

    case, z, bc, (u, v, w, p), d = _setup(name)
    bc.EnforceVelocityBC(u, v, w, None)
    bc.EnforcePressureBC(p, None)
    torch.cuda.synchronize()
    lists = dict(z)
    lists["ring_value"] = np.zeros_like(z["ring_value"])
    ru, rv, rw, rp = cpu.bc_replay(lists, z["u_in"], z["v_in"], z["w_in"], z["p_in"], with_velocity_function=False)
    hu, hv, hw, hp = _host([u, v, w, p])
    assert np.array_equal(hu, ru) and np.array_equal(hv, rv) and np.array_equal(hp, rp)
    assert np.array_equal(hw, rw)
    bc.close()


def test_replay_in_a_cuda_graph(nb):
    import torch

    name = [n for n in NAMES if "channel" in n][0]
    case, z, bc, (u, v, w, p), d = _setup(name)
    pv, rv = d(z["presc_value"]), d(z["ring_value"])
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        bc.EnforceVelocityBC(u, v, w, pv, stream=s)
        bc.EnforcePressureBC(p, rv, stream=s)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s, capture_error_mode="thread_local"):
        bc.EnforceVelocityBC(u, v, w, pv, stream=s)
        bc.EnforcePressureBC(p, rv, stream=s)
    rng = np.random.default_rng(5)
    for _ in range(2):
        ins = [rng.normal(size=len(z[k])) for k in ("u_in", "v_in", "w_in", "p_in")]
        for t, a in zip((u, v, w, p), ins):
            t.copy_(torch.from_numpy(a))
        graph.replay()
        torch.cuda.synchronize()
        ref = cpu.bc_replay(dict(z), *ins)
        for got, want in zip(_host([u, v, w, p]), ref):
            assert np.array_equal(got, want)
    del graph
    bc.close()
