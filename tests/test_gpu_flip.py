"""FLIP's re-labelling from particles on the B200 (nereus_b200_update_fluid_cells[_device]) against the reference's
own FLIP{2,3}D::UpdateFluidCells (tests/golden/flip_relabel_*.npz) and the oracle's restatement of it: the labels
must agree byte for byte, and the pressure step on the new labels must give the reference's projection."""
import ctypes

import numpy as np
import pytest

from conftest import flip_golden_names, load_golden
from nereus_cfd_b200 import capi, workloads as W
from nereus_cfd_b200.pressure import MACGrid, PressureSolver
from oracle import cpu

pytestmark = pytest.mark.gpu
NAMES = flip_golden_names()


def _origin(grid):
    return [ax.face[0] for ax in grid.axes]


def device_relabel(nb, grid, types, xyz, origin, scratch_bytes=None):
    """The device form on torch tensors; xyz rows may be wider than 3 (x, y, z at columns 0..2)."""
    import torch

    t = torch.from_numpy(np.ascontiguousarray(types, dtype=np.uint8).reshape(-1)).to("cuda")
    pos = torch.from_numpy(np.ascontiguousarray(xyz, dtype=np.float64)).to("cuda")
    count, stride = (pos.shape[0], pos.shape[1]) if pos.numel() else (0, 3)
    nz = grid.Nz if grid.dim == 3 else 1
    full = nb.nereus_b200_update_fluid_cells_scratch_bytes(grid.dim, grid.Nx, grid.Ny, nz)
    sb = full if scratch_bytes is None else scratch_bytes
    scratch = torch.zeros(max(sb, 16) // 4 + 1, dtype=torch.int32, device="cuda")
    skipped = torch.full((1,), -5, dtype=torch.int64, device="cuda")
    base = pos.data_ptr()
    st = nb.nereus_b200_update_fluid_cells_device(
        torch.cuda.current_device(), grid.dim, grid.Nx, grid.Ny, nz, origin[0], origin[1],
        origin[2] if grid.dim == 3 else 0.0, grid.dh, ctypes.c_void_p(base), ctypes.c_void_p(base + 8),
        ctypes.c_void_p(base + 16) if grid.dim == 3 else None, count, stride, ctypes.c_void_p(t.data_ptr()),
        ctypes.c_void_p(scratch.data_ptr()), sb, ctypes.c_void_p(skipped.data_ptr()),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    capi.check(st)
    torch.cuda.synchronize()
    return t.cpu().numpy(), int(skipped.item())


@pytest.mark.parametrize("name", NAMES)
def test_host_form_matches_reference(nb, name):
    case, meta, z = load_golden(name)
    out, skipped = capi.update_fluid_cells(case.grid, z["types_in"], z["xyz"], meta["origin"], meta["dh"])
    assert skipped == 0
    assert np.array_equal(out, z["types"])


@pytest.mark.parametrize("name", NAMES)
def test_reference_particle_rows(nb, name):
    """The reference's own Particle array: 7 doubles a particle (isActive padded to 8 bytes, x, y, z, u, v, w)."""
    case, meta, z = load_golden(name)
    n = z["xyz"].shape[0]
    rows = np.zeros((n, 7))
    rows[:, 0] = np.nan  # the isActive word is never read
    rows[:, 1:4] = z["xyz"]
    rows[:, 4:] = 123.0
    g = case.grid
    out = z["types_in"].copy()
    skipped = ctypes.c_int64(-1)
    base = rows.ctypes.data
    o = meta["origin"]
    capi.check(nb.nereus_b200_update_fluid_cells(
        g.dim, g.Nx, g.Ny, g.Nz if g.dim == 3 else 1, o[0], o[1], o[2], meta["dh"], ctypes.c_void_p(base + 8),
        ctypes.c_void_p(base + 16), ctypes.c_void_p(base + 24) if g.dim == 3 else None, n, 7,
        capi.ptr(out, capi._u8), ctypes.byref(skipped)))
    assert skipped.value == 0 and np.array_equal(out, z["types"])


@pytest.mark.parametrize("scratch", [None, 16, 40])
@pytest.mark.parametrize("name", NAMES)
def test_device_form_matches_reference(nb, name, scratch):
    """Full scratch, none beyond the header (every undecided cell settled by passes over the whole interior), and a
    list too short for the undecided cells."""
    case, meta, z = load_golden(name)
    out, skipped = device_relabel(nb, case.grid, z["types_in"], z["xyz"], meta["origin"], scratch)
    assert skipped == 0
    assert np.array_equal(out, z["types"])


CASES = [(W.flip_tank_3d, {"n": 40, "seed": 61}, 0.03, 4), (W.flip_tank_3d, {"n": 33, "seed": 62}, 0.35, 2),
         (W.flip_tank_3d, {"n": 24, "seed": 63}, 0.7, 1), (W.flip_tank_2d, {"n": 150, "seed": 64}, 0.3, 3),
         (W.flip_tank_2d, {"n": 37, "seed": 65}, 0.6, 2), (W.flip_tank_3d, {"n": 128, "seed": 66}, 0.2, 2)]


@pytest.mark.parametrize("builder,kwargs,holes,ppc", CASES)
def test_random_clouds_match_oracle(nb, builder, kwargs, holes, ppc):
    case = builder(**kwargs)
    g = case.grid
    t = cpu.label_cells(g, case.scene)
    xyz = W.flip_particles(case, t, 100 + kwargs["seed"], ppc, hole_fraction=holes)
    org = _origin(g)
    ref, ref_sk = cpu.update_fluid_cells(g, t, xyz, org)
    for scratch in (None, 16):
        out, sk = device_relabel(nb, g, t, xyz, org, scratch)
        assert sk == ref_sk
        assert np.array_equal(out, ref)


def test_out_of_range_particles_and_empty_cloud(nb):
    case = W.flip_tank_3d(n=12, seed=70)
    g = case.grid
    t = cpu.label_cells(g, case.scene)
    org = _origin(g)
    dh = g.dh
    good = W.flip_particles(case, t, 71, 2)
    bad = np.array([[org[0] - 1.5 * dh, org[1] + 3.5 * dh, org[2] + 3.5 * dh],
                    [np.nan, org[1] + 3.5 * dh, org[2] + 3.5 * dh],
                    [org[0] + 3.5 * dh, -np.inf, org[2] + 3.5 * dh],
                    [org[0] + 3.5 * dh, org[1] + 3.5 * dh, np.inf],
                    [1e300, 1e300, 1e300]])
    xyz = np.concatenate([good, bad])
    ref, ref_sk = cpu.update_fluid_cells(g, t, xyz, org)
    assert ref_sk == 3
    for fn in (lambda: capi.update_fluid_cells(g, t, xyz, org), lambda: device_relabel(nb, g, t, xyz, org)):
        out, sk = fn()
        assert sk == ref_sk and np.array_equal(out, ref)
    ref0, _ = cpu.update_fluid_cells(g, t, np.zeros((0, 3)), org)
    out0, sk0 = capi.update_fluid_cells(g, t, np.zeros((0, 3)), org)
    assert sk0 == 0 and np.array_equal(out0, ref0)
    assert not (out0 == W.FLUID).any()


def test_device_form_replays_in_a_cuda_graph(nb):
    import torch

    case = W.flip_tank_3d(n=20, seed=72)
    g = case.grid
    t0 = cpu.label_cells(g, case.scene)
    org = _origin(g)
    xyz_a = W.flip_particles(case, t0, 73, 2, hole_fraction=0.3)
    xyz_b = W.flip_particles(case, t0, 74, 2, hole_fraction=0.3)[: xyz_a.shape[0]]
    n = min(xyz_a.shape[0], xyz_b.shape[0])
    xyz_a, xyz_b = xyz_a[:n], xyz_b[:n]
    t_in = torch.from_numpy(t0).to("cuda")
    t = t_in.clone()
    pos = torch.from_numpy(np.ascontiguousarray(xyz_a)).to("cuda")
    sb = nb.nereus_b200_update_fluid_cells_scratch_bytes(3, g.Nx, g.Ny, g.Nz)
    scratch = torch.zeros(sb // 4 + 1, dtype=torch.int32, device="cuda")
    skipped = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = torch.cuda.Stream()
    base = pos.data_ptr()

    def call():
        capi.check(nb.nereus_b200_update_fluid_cells_device(
            torch.cuda.current_device(), 3, g.Nx, g.Ny, g.Nz, org[0], org[1], org[2], g.dh, ctypes.c_void_p(base),
            ctypes.c_void_p(base + 8), ctypes.c_void_p(base + 16), n, 3, ctypes.c_void_p(t.data_ptr()),
            ctypes.c_void_p(scratch.data_ptr()), sb, ctypes.c_void_p(skipped.data_ptr()),
            ctypes.c_void_p(s.cuda_stream)))

    with torch.cuda.stream(s):
        call()  # outside capture first
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s, capture_error_mode="thread_local"):
        call()
    for xyz in (xyz_b, xyz_a):
        pos.copy_(torch.from_numpy(np.ascontiguousarray(xyz)))
        t.copy_(t_in)
        graph.replay()
        torch.cuda.synchronize()
        ref, _ = cpu.update_fluid_cells(g, t0, xyz, org)
        assert np.array_equal(t.cpu().numpy(), ref)
    del graph


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("name", NAMES)
def test_relabel_then_projection_matches_reference(nb, name, precision):
    """The FLIP step's label update and pressure projection, both on the B200, against the reference's."""
    case, meta, z = load_golden(name)
    g = case.grid
    types, _ = capi.update_fluid_cells(g, z["types_in"], z["xyz"], meta["origin"], meta["dh"])
    m = MACGrid(g, types, z["u"].copy(), z["v"].copy(), z["w"].copy(), z["p_in"].copy(), meta["rho"], meta["dt"])
    s = PressureSolver(precision)
    r = s.SolvePressure(m, tol=1e-10, needs_compat=meta["needs_compat"])
    assert r.status == capi.NB_OK and r.n == meta["n"]
    assert np.array_equal(s.IDP(), z["idp"])
    s.DestroyPressureSolver()
    idp = z["idp"]
    x = m.p[idp >= 0][np.argsort(idp[idp >= 0])]
    assert np.linalg.norm(x - z["x"]) <= 1e-6 * np.linalg.norm(z["x"])
    scale = max(np.abs(z["u"]).max(), np.abs(z["v"]).max())
    assert np.abs(m.u - z["u_out"]).max() <= 1e-6 * scale
    assert np.abs(m.v - z["v_out"]).max() <= 1e-6 * scale
    if g.dim == 3:
        assert np.abs(m.w - z["w_out"]).max() <= 1e-6 * scale
