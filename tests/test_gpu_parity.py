"""Parity of the B200 path with the reference, through the C ABI, on every golden fixture (tests/golden, written by
the reference's own pressure path) and against the oracle.

Bars (written here, per the specification of this path):
  * cell labelling, IDP numbering, the assembled stencil (CSR values) and the raw right-hand side: bit-exact;
  * the velocity correction of a given pressure: bit-exact;
  * the solve: relative residual ||b - A x|| / ||b|| <= the requested tolerance, mean-free pressure within
    1e-6 relative L2 of the reference's Eigen-CG solution, post-projection max |div u| within 10x of the
    reference's when both solve to the same tolerance;
  * repeating a solve is bit-identical (tests/suite_pressure.cpp:119-141).
"""
import ctypes

import numpy as np
import pytest

from conftest import golden_names, load_golden
from nereus_cfd_b200 import capi, workloads as W
from nereus_cfd_b200.pressure import MACGrid, PressureSolver

pytestmark = pytest.mark.gpu
NAMES = golden_names()
PRECISIONS = ["mixed", "fp64"]


def mac_from_golden(case, meta, z):
    g = case.grid
    return MACGrid(g, z["types"].copy(), z["u"].copy(), z["v"].copy(), z["w"].copy(), z["p_in"].copy(),
                   meta["rho"], meta["dt"])


@pytest.mark.parametrize("name", NAMES)
def test_labels_bit_exact(nb, name):
    case, meta, z = load_golden(name)
    assert np.array_equal(capi.label_cells(case.grid, case.scene), z["types"])


@pytest.mark.parametrize("name", NAMES)
def test_idp_and_matrix_bit_exact(nb, name):
    case, meta, z = load_golden(name)
    s = PressureSolver("fp64")
    s.InitializePressureSolver(mac_from_golden(case, meta, z))
    assert s.SystemSize() == meta["n"]
    assert np.array_equal(s.IDP(), z["idp"])
    rowptr, col, val, singular = s.ExportMatrix()
    assert singular == meta["singular"]
    assert np.array_equal(rowptr, z["rowptr"])
    assert np.array_equal(col, z["col"])
    assert np.array_equal(val, z["val"])
    s.DestroyPressureSolver()


@pytest.mark.parametrize("name", NAMES)
def test_rhs_bit_exact(nb, name):
    case, meta, z = load_golden(name)
    s = PressureSolver("fp64")
    m = mac_from_golden(case, meta, z)
    s.InitializePressureSolver(m)
    assert np.array_equal(s.Rhs(m), z["b_raw"])
    s.DestroyPressureSolver()


@pytest.mark.parametrize("name", NAMES)
def test_projection_of_reference_pressure_bit_exact(nb, name):
    case, meta, z = load_golden(name)
    s = PressureSolver("fp64")
    m = mac_from_golden(case, meta, z)
    s.InitializePressureSolver(m)
    u, v = m.u.copy(), m.v.copy()
    w = m.w.copy() if m.w.size else np.zeros(1)
    p = np.ascontiguousarray(z["p"])
    capi.check(s.lib.nereus_b200_project_velocity(s.ctx, capi.ptr(u), capi.ptr(v), capi.ptr(w), capi.ptr(p),
                                                  meta["rho"], meta["dt"]))
    assert np.array_equal(u, z["u_out"])
    assert np.array_equal(v, z["v_out"])
    if m.w.size:
        assert np.array_equal(w, z["w_out"])
    s.DestroyPressureSolver()


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("name", NAMES)
def test_solve_and_project_against_reference(nb, name, precision):
    case, meta, z = load_golden(name)
    tol = meta["tol"]
    s = PressureSolver(precision)
    m = mac_from_golden(case, meta, z)
    r = s.SolvePressure(m, tol=tol, needs_compat=meta["needs_compat"])
    assert r.status == capi.NB_OK, r.as_dict()
    assert r.n == meta["n"]
    assert r.rel_res <= tol
    if meta["n"]:
        idp = z["idp"]
        x = m.p[idp >= 0][np.argsort(idp[idp >= 0])]
        xr = z["x"]
        if meta["singular"]:
            x, xr = x - x.mean(), xr - xr.mean()
        err = np.linalg.norm(x - xr) / max(np.linalg.norm(xr), 1e-300)
        assert err <= 1e-6, err
        # Dirichlet ring cells and interior non-unknowns exactly as the reference left them; the copied ring cells
        # carry an interior value, so they agree to the solution's tolerance
        g = case.grid
        t = z["types"].reshape(g.shape)
        ring = np.ones(g.shape, dtype=bool)
        ring[1:-1, 1:-1, (slice(1, -1) if g.dim == 3 else slice(None))] = False
        ring = ring.reshape(-1)
        fixed = (idp < 0) & (~ring | np.isin(z["types"], [W.EMPTY, W.PRESSURE]))
        copied = (idp < 0) & ring & ~np.isin(z["types"], [W.EMPTY, W.PRESSURE])
        assert np.array_equal(m.p[fixed], z["p"][fixed])
        scale = max(np.abs(z["p"]).max(), 1e-300)
        assert np.abs(m.p[copied] - z["p"][copied]).max(initial=0.0) <= 1e-6 * scale
        del t
        assert r.max_div <= 10.0 * max(meta["max_div"], 1e-300) + 1e-12, (r.max_div, meta["max_div"])
    else:
        assert np.array_equal(m.u, z["u_out"]) and np.array_equal(m.v, z["v_out"])
    s.DestroyPressureSolver()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_repeat_solve_is_bit_identical(nb, precision):
    case, meta, z = load_golden("sphere_outlet_3d_12")
    s = PressureSolver(precision)
    m1, m2 = mac_from_golden(case, meta, z), mac_from_golden(case, meta, z)
    s.SolvePressure(m1, tol=1e-10)
    s.SolvePressure(m2, tol=1e-10)
    assert np.array_equal(m1.p, m2.p) and np.array_equal(m1.u, m2.u)
    s.DestroyPressureSolver()


@pytest.mark.parametrize("name,bar", [("dirichlet_linear_2d_40", 1e-7), ("dirichlet_linear_3d_20", 1e-8)])
def test_known_answer_linear_field(nb, name, bar):
    """tests/suite_pressure.cpp:166-169, 230: the linear Dirichlet field is reproduced to the reference's bars."""
    case, meta, z = load_golden(name)
    g = case.grid
    s = PressureSolver("mixed")
    m = mac_from_golden(case, meta, z)
    r = s.SolvePressure(m, tol=meta["tol"])
    assert r.status == capi.NB_OK
    p = m.p.reshape(g.shape)
    xs, ys = g.axes[0].centre, g.axes[1].centre
    ks = range(1, g.Nz - 1) if g.dim == 3 else [0]
    worst = max(abs(p[i, j, k] - (0.3 + 1.1 * xs[j] - 0.7 * ys[i]))
                for i in range(1, g.Ny - 1) for j in range(1, g.Nx - 1) for k in ks)
    assert worst < bar
    s.DestroyPressureSolver()


def test_split_steps_equal_fused(nb):
    """The pressure step then the projection step gives what the fused call gives."""
    case, meta, z = load_golden("stretched_cylinder_3d_24x16x16")
    s = PressureSolver("fp64")
    m1, m2 = mac_from_golden(case, meta, z), mac_from_golden(case, meta, z)
    s.SolvePressure(m1, tol=1e-10)
    r = capi.Result()
    capi.check(s.lib.nereus_b200_solve_pressure(s.ctx, capi.ptr(m2.u), capi.ptr(m2.v), capi.ptr(m2.w),
                                                capi.ptr(m2.p), m2.rho, m2.dt, 0, 0, 1e-10, ctypes.byref(r)))
    assert np.array_equal(m1.p, m2.p)
    capi.check(s.lib.nereus_b200_project_velocity(s.ctx, capi.ptr(m2.u), capi.ptr(m2.v), capi.ptr(m2.w),
                                                  capi.ptr(m2.p), m2.rho, m2.dt))
    assert np.array_equal(m1.u, m2.u) and np.array_equal(m1.v, m2.v) and np.array_equal(m1.w, m2.w)
    s.DestroyPressureSolver()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_solve_laplacian(nb, precision):
    """SolveLaplacian: L x = f with the pressure matrix, A x = V f (PressureSolver3D.cpp:355-371)."""
    from oracle import cpu

    case, meta, z = load_golden("stretched_cylinder_3d_24x16x16")
    s = PressureSolver(precision)
    m = mac_from_golden(case, meta, z)
    s.InitializePressureSolver(m)
    n = s.SystemSize()
    ok, x = s.SolveLaplacian(m, np.zeros(n + 1))
    assert not ok and x is None
    f = W.normals(99, n)
    ok, x = s.SolveLaplacian(m, f, tol=1e-10)
    assert ok
    asm = cpu.assemble(cpu.GridView(case.grid, z["types"]))
    g = case.grid
    vol = np.empty(n)
    t = z["types"].reshape(g.shape)
    idp = z["idp"].reshape(g.shape)
    for i, j, k in zip(*np.nonzero(idp >= 0)):
        vol[idp[i, j, k]] = g.axes[0].size[j] * g.axes[1].size[i] * g.axes[2].size[k]
    b = f * vol
    assert cpu.residual_norm(asm, b, x) / np.linalg.norm(b) <= 1e-10
    s.DestroyPressureSolver()


def test_bad_inputs_are_reported(nb):
    case, meta, z = load_golden("sphere_outlet_3d_12")
    s = PressureSolver("mixed")
    m = mac_from_golden(case, meta, z)
    s.InitializePressureSolver(m)
    bad = m.types.copy()
    bad[5] = 9
    with pytest.raises(capi.NBError) as e:
        s.EnsureSystem(MACGrid(m.grid, bad, m.u, m.v, m.w, m.p))
    assert e.value.status == capi.NB_BAD_INPUT
    r = capi.Result()
    st = s.lib.nereus_b200_project(s.ctx, capi.ptr(m.u), capi.ptr(m.v), capi.ptr(m.w), capi.ptr(m.p), 1.0, 1e-3,
                                   capi.SCHEME_INCREMENTAL, 0, 1e-8, ctypes.byref(r))
    assert st == capi.NB_BAD_INPUT
    st = s.lib.nereus_b200_project(s.ctx, capi.ptr(m.u), capi.ptr(m.v), capi.ptr(m.w), capi.ptr(m.p), -1.0, 1e-3,
                                   0, 0, 1e-8, ctypes.byref(r))
    assert st == capi.NB_BAD_INPUT
    s.DestroyPressureSolver()


def test_iteration_cap_reports_not_converged(nb):
    case, meta, z = load_golden("stretched_cylinder_3d_24x16x16")
    s = PressureSolver("fp64", max_iters=1, max_outer=1)
    m = mac_from_golden(case, meta, z)
    r = s.SolvePressure(m, tol=1e-14)
    assert r.status == capi.NB_NOT_CONVERGED
    assert np.all(np.isfinite(m.p))
    s.DestroyPressureSolver()
