"""The three FP32 kernel families of the mixed-precision inner solve against each other and the reference.

pair_kernels = 0 (per-cell kernels), 1 (cell pairs in the grid layout), 2 (the colour-split layout, the default):
the same V-cycle up to FP32 rounding, so every family meets the parity bars of the solve (relative residual <= the
tolerance, mean-free pressure within 1e-6 rel-L2 of the reference's solution), and on grids deep enough for several
colour-split levels the split solution agrees with the cell-pair one to the solve's tolerance.
"""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from nereus_cfd_b200 import capi, workloads as W
from nereus_cfd_b200.pressure import MACGrid, PressureSolver

pytestmark = pytest.mark.gpu
FAMILIES = [0, 1, 2]
NAMES_3D = [n for n in golden_names() if "_3d_" in n]


def mac_from_golden(case, meta, z):
    return MACGrid(case.grid, z["types"].copy(), z["u"].copy(), z["v"].copy(), z["w"].copy(), z["p_in"].copy(),
                   meta["rho"], meta["dt"])


@pytest.mark.parametrize("family", FAMILIES)
@pytest.mark.parametrize("name", NAMES_3D)
def test_family_against_reference(nb, name, family):
    case, meta, z = load_golden(name)
    s = PressureSolver("mixed", pair_kernels=family)
    m = mac_from_golden(case, meta, z)
    r = s.SolvePressure(m, tol=meta["tol"], needs_compat=meta["needs_compat"])
    assert r.status == capi.NB_OK, r.as_dict()
    assert r.rel_res <= meta["tol"]
    if meta["n"]:
        idp = z["idp"]
        x = m.p[idp >= 0][np.argsort(idp[idp >= 0])]
        xr = z["x"]
        if meta["singular"]:
            x, xr = x - x.mean(), xr - xr.mean()
        assert np.linalg.norm(x - xr) / max(np.linalg.norm(xr), 1e-300) <= 1e-6
    s.DestroyPressureSolver()


def closed_box_3d(n):
    g = W.uniform_grid(3, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    sph = W.Region(W.REGION_SOLID, W.PRIM_SPHERE, (0.4, 0.5, 0.6), radius=0.2)
    return W.Case("closed_box_3d_%d" % n, g, W.walls_scene(3, regions=[sph]), 9, needs_compat=True, tol=1e-9)


CASES = {
    "sphere_outlet_48": lambda: W.sphere_outlet_3d(48),
    "flip_tank_40": lambda: W.flip_tank_3d(40),
    "stretched_cylinder_48x32x32": lambda: W.stretched_cylinder_3d(48, 32, 32),
    "closed_box_40": lambda: closed_box_3d(40),
    # 30 x 36 x 26 interior cells: odd coarse sizes along x and z (15, 13), rows padded to the split's multiple of 4
    "sphere_outlet_30x36x26": lambda: W.Case(
        "sphere_outlet_30x36x26", W.uniform_grid(3, (0.0, 1.0, 0.0, 1.2, 0.0, 26.0 / 30.0), 30),
        W.sphere_outlet_3d(8).scene, 2),
}


def solve(case, family, tol):
    g = case.grid
    types = capi.label_cells(g, case.scene)
    u, v, w = W.face_velocities(g, types, case.seed, case.velocity_rule, case.fp32_velocity)
    m = MACGrid(g, types.copy(), u.copy(), v.copy(), w.copy(), np.zeros(g.cells), case.rho, case.dt)
    s = PressureSolver("mixed", pair_kernels=family)
    r = s.SolvePressure(m, tol=tol, needs_compat=case.needs_compat)
    s.DestroyPressureSolver()
    return r, m, types


@pytest.mark.parametrize("name", sorted(CASES))
def test_split_agrees_with_pairs(nb, name):
    case = CASES[name]()
    tol = 1e-9
    r2, m2, types = solve(case, 2, tol)
    r1, m1, _ = solve(case, 1, tol)
    assert r2.status == capi.NB_OK and r1.status == capi.NB_OK
    assert r2.rel_res <= tol and r1.rel_res <= tol
    assert r2.levels >= 3
    unk = np.zeros(case.grid.shape, dtype=bool)
    unk[1:-1, 1:-1, 1:-1] = (types.reshape(case.grid.shape) == W.FLUID)[1:-1, 1:-1, 1:-1]
    unk = unk.reshape(-1)
    p1, p2 = m1.p[unk], m2.p[unk]
    if r1.singular:
        p1, p2 = p1 - p1.mean(), p2 - p2.mean()
    assert np.linalg.norm(p2 - p1) / max(np.linalg.norm(p1), 1e-300) <= 1e-6
    # the same preconditioner up to FP32 rounding: about the same iterations
    assert abs(r2.iters_inner - r1.iters_inner) <= 2 + r1.iters_inner // 5, (r2.iters_inner, r1.iters_inner)


def test_split_repeat_is_bit_identical(nb):
    case = W.sphere_outlet_3d(32)
    _, a, _ = solve(case, 2, 1e-10)
    _, b, _ = solve(case, 2, 1e-10)
    assert np.array_equal(a.p, b.p) and np.array_equal(a.u, b.u)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_device_loop_equals_host_loop(nb, precision):
    """The CG loop as one graph with a device-side WHILE condition (use_graphs = 2), one graph per iteration
    (use_graphs = 1) and plain launches iteration by iteration from the host (use_graphs = 0) run the same kernels in
    the same order: the same iterations and the same bits."""
    case = W.sphere_outlet_3d(40)
    g = case.grid
    types = capi.label_cells(g, case.scene)
    u, v, w = W.face_velocities(g, types, case.seed, case.velocity_rule, case.fp32_velocity)
    out = []
    for graphs in (2, 1, 0):
        m = MACGrid(g, types.copy(), u.copy(), v.copy(), w.copy(), np.zeros(g.cells), case.rho, case.dt)
        s = PressureSolver(precision, use_graphs=graphs)
        r = s.SolvePressure(m, tol=1e-9)
        assert r.status == capi.NB_OK and r.rel_res <= 1e-9
        # a second solve on the same context replays the loop built by the first
        m2 = MACGrid(g, types.copy(), u.copy(), v.copy(), w.copy(), np.zeros(g.cells), case.rho, case.dt)
        r2 = s.SolvePressure(m2, tol=1e-9)
        s.DestroyPressureSolver()
        assert np.array_equal(m.p, m2.p) and r.iters_inner == r2.iters_inner
        out.append((r.iters_inner, r.iters_outer, m.p, m.u))
    for o in out[1:]:
        assert out[0][:2] == o[:2]
        assert np.array_equal(out[0][2], o[2]) and np.array_equal(out[0][3], o[3])


def test_device_loop_stops_at_the_iteration_cap(nb):
    case = W.sphere_outlet_3d(32)
    g = case.grid
    types = capi.label_cells(g, case.scene)
    u, v, w = W.face_velocities(g, types, case.seed, case.velocity_rule, case.fp32_velocity)
    m = MACGrid(g, types.copy(), u.copy(), v.copy(), w.copy(), np.zeros(g.cells), case.rho, case.dt)
    s = PressureSolver("fp64", max_iters=2, max_outer=1)
    r = s.SolvePressure(m, tol=1e-12)
    s.DestroyPressureSolver()
    assert r.status == capi.NB_NOT_CONVERGED
    assert r.iters_inner == 2


@pytest.mark.parametrize("name", ["closed_box_2d", "stretched_cylinder_3d", "flip_tank_3d"])
def test_device_refinement_loop_equals_host_loop(nb, name):
    """The mixed solve as one graph (use_graphs = 2: the refinement passes in a WHILE node around the CG loop's WHILE
    node) and the refinement loop on the host (use_graphs = 1): the same passes, iterations and bits, on a singular
    2D box (compatibility on), a stretched 3D channel and a free-surface tank."""
    case = {"closed_box_2d": lambda: W.closed_box_2d(48, seed=3),
            "stretched_cylinder_3d": lambda: W.stretched_cylinder_3d(24, 16, 16, seed=4),
            "flip_tank_3d": lambda: W.flip_tank_3d(30, seed=5)}[name]()
    g = case.grid
    types = capi.label_cells(g, case.scene)
    u, v, w = W.face_velocities(g, types, case.seed, case.velocity_rule, case.fp32_velocity)
    out = []
    for graphs in (2, 1):
        s = PressureSolver("mixed", use_graphs=graphs)
        for rep in range(2):
            m = MACGrid(g, types.copy(), u.copy(), v.copy(), w.copy(), np.zeros(g.cells), case.rho, case.dt)
            r = s.SolvePressure(m, tol=1e-10, needs_compat=case.needs_compat)
            assert r.status == capi.NB_OK and r.rel_res <= 1e-10
            out.append((r.iters_inner, r.iters_outer, r.rel_res, m.p, m.u, m.v))
        s.DestroyPressureSolver()
    for o in out[1:]:
        assert out[0][:3] == o[:3]
        for a, b in zip(out[0][3:], o[3:]):
            assert np.array_equal(a, b)


def test_device_refinement_loop_limits(nb):
    """The device-side refinement loop stops at max_outer passes with NOT_CONVERGED, and a zero right-hand side needs
    no pass at all."""
    case = W.sphere_outlet_3d(24, seed=6)
    g = case.grid
    types = capi.label_cells(g, case.scene)
    u, v, w = W.face_velocities(g, types, case.seed, case.velocity_rule, case.fp32_velocity)
    s = PressureSolver("mixed", max_outer=1)
    m = MACGrid(g, types.copy(), u.copy(), v.copy(), w.copy(), np.zeros(g.cells), case.rho, case.dt)
    r = s.SolvePressure(m, tol=1e-14)
    assert r.status == capi.NB_NOT_CONVERGED and r.iters_outer == 1 and r.rel_res > 1e-14
    z = MACGrid(g, types.copy(), np.zeros_like(u), np.zeros_like(v), np.zeros_like(w), np.zeros(g.cells), case.rho,
                case.dt)
    r0 = s.SolvePressure(z, tol=1e-8)
    s.DestroyPressureSolver()
    assert r0.status == capi.NB_OK and r0.iters_outer == 0 and r0.iters_inner == 0 and r0.rel_res == 0.0
    assert not np.any(z.p[types == W.FLUID])
