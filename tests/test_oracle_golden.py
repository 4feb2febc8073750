"""The oracle pinned against the reference: every fixture under tests/golden was written by the NEREUS reference's own
pressure path (tests/golden/make_golden.py). Cell types, spacing tables, IDP numbering, the CSR matrix and the raw
right-hand side must be bit-exact; the CG solution within its tolerance; the projection of the reference's pressure
bit-exact. The known-answer cases repeat tests/suite_pressure.cpp's checks (a linear Dirichlet field is exact)."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from nereus_cfd_b200 import workloads as W
from oracle import cpu

NAMES = golden_names()


def test_fixtures_present():
    assert len(NAMES) >= 9


@pytest.mark.parametrize("name", NAMES)
def test_tables_and_labels(name):
    case, meta, z = load_golden(name)
    g = case.grid
    for a in range(3):
        assert np.array_equal(g.width_tables()[a], z["width%d" % a]), "width table %d" % a
        assert np.array_equal(g.gap_tables()[a], z["gap%d" % a]), "gap table %d" % a
        assert np.array_equal(g.axes[a].centre, z["centre%d" % a][1:-1])  # the padded table without its ghosts
    types = cpu.label_cells(g, case.scene)
    assert np.array_equal(types, z["types"])


@pytest.mark.parametrize("name", NAMES)
def test_assembly_bit_exact(name):
    case, meta, z = load_golden(name)
    gv = cpu.GridView(case.grid, z["types"])
    asm = cpu.assemble(gv)
    assert asm.n == meta["n"]
    assert asm.singular == meta["singular"]
    assert np.array_equal(asm.idp, z["idp"])
    assert np.array_equal(asm.rowptr, z["rowptr"])
    assert np.array_equal(asm.col, z["col"])
    assert np.array_equal(asm.val, z["val"])  # bit-exact FP64 coefficients


@pytest.mark.parametrize("name", NAMES)
def test_rhs_bit_exact(name):
    case, meta, z = load_golden(name)
    g = case.grid
    gv = cpu.GridView(g, z["types"])
    asm = cpu.assemble(gv)
    p = cpu.ring_replay(g, z["types"], z["p_in"])
    b = cpu.rhs(gv, asm, z["u"], z["v"], z["w"], p, meta["rho"], meta["dt"])
    assert np.array_equal(b, z["b_raw"])
    if meta["needs_compat"] and meta["singular"] and asm.n:
        bc = cpu.compat(b)
        assert np.array_equal(bc, z["b"])  # the same serial summation order
    else:
        assert np.array_equal(b, z["b"])


@pytest.mark.parametrize("name", NAMES)
def test_solution_and_projection(name):
    case, meta, z = load_golden(name)
    g = case.grid
    r = cpu.solve_projection(g, z["types"], z["u"], z["v"], z["w"], z["p_in"], meta["rho"], meta["dt"],
                             meta["needs_compat"], meta["tol"])
    assert r.iters == meta["iters"]
    if meta["n"]:
        xr, xo = z["x"], r.x
        if meta["singular"]:
            xr, xo = xr - xr.mean(), xo - xo.mean()
        assert np.linalg.norm(xo - xr) <= 1e-9 * max(np.linalg.norm(xr), 1e-300)
        assert r.rel_res <= meta["tol"] * 1.0001
    # the projection applied to the reference's own pressure reproduces its velocities exactly
    gv = cpu.GridView(g, z["types"])
    uu, vv = z["u"].copy(), z["v"].copy()
    ww = z["w"].copy() if z["w"].size else np.zeros(1)
    p = np.ascontiguousarray(z["p"])
    cpu.lib().or_project(gv.ref, cpu._p(uu, cpu._dp), cpu._p(vv, cpu._dp), cpu._p(ww, cpu._dp), cpu._p(p, cpu._dp),
                         meta["rho"], meta["dt"])
    assert np.array_equal(uu, z["u_out"])
    assert np.array_equal(vv, z["v_out"])
    if z["w"].size:
        assert np.array_equal(ww, z["w_out"])


@pytest.mark.parametrize("name", NAMES)
def test_ring_replay_matches_reference(name):
    """Scatter + EnforcePressureBC: the reference's x scattered and the ring replayed gives its p exactly."""
    case, meta, z = load_golden(name)
    g = case.grid
    gv = cpu.GridView(g, z["types"])
    p = cpu.ring_replay(g, z["types"], z["p_in"])
    xs = z["x"] if z["x"].size else np.zeros(1)
    cpu.lib().or_scatter(gv.ref, cpu._p(z["idp"], cpu._ip), cpu._p(np.ascontiguousarray(xs), cpu._dp),
                         cpu._p(p, cpu._dp))
    cpu.lib().or_ring_replay(gv.ref, cpu._p(p, cpu._dp))
    assert np.array_equal(p, z["p"])


@pytest.mark.parametrize("name,bar", [("dirichlet_linear_2d_40", 1e-7), ("dirichlet_linear_3d_20", 1e-8)])
def test_known_answer_linear_field(name, bar):
    """tests/suite_pressure.cpp:166-169 (2D, < 1e-7) and :230 (3D, < 1e-8): p = 0.3 + 1.1x - 0.7y is exact."""
    case, meta, z = load_golden(name)
    g = case.grid
    r = cpu.solve_projection(g, z["types"], z["u"], z["v"], z["w"], z["p_in"], meta["rho"], meta["dt"], False,
                             meta["tol"])
    p = r.p.reshape(g.shape)
    xs, ys = g.axes[0].centre, g.axes[1].centre
    worst = 0.0
    for i in range(1, g.Ny - 1):
        for j in range(1, g.Nx - 1):
            exact = 0.3 + 1.1 * xs[j] - 0.7 * ys[i]
            for k in range(1, g.Nz - 1) if g.dim == 3 else [0]:
                worst = max(worst, abs(p[i, j, k] - exact))
    assert worst < bar
    assert np.abs(p).max() > 0.1


def test_velocity_generator_is_seeded():
    a = W.normals(123, 1001)
    b = W.normals(123, 1001)
    assert np.array_equal(a, b)
    assert abs(a.mean()) < 0.15 and abs(a.std() - 1.0) < 0.1
    assert not np.array_equal(a, W.normals(124, 1001))
