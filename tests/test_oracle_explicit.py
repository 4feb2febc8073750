"""The EXPLICIT method's own pressure step (src/Methods/Explicit/Explicit2D.cpp:48-120: SOR sweeps on a 5-point
stencil with coefficient 1 toward fluid and 2 toward pressure-outlet cells, the mean removed when no outlet exists)
and its projection (:106-120) solve the same system as the shared pressure path on uniform 2D scenes whose Dirichlet
cells lie on the ring: the outlet coefficient 2 is the shared ring factor. So a NEREUS build can route EXPLICIT's
pressure and projection steps through this backend's project call.

The fixtures (tests/golden/explicit_*.npz) hold what the reference's Explicit2D::Pressure and ::Projection computed,
SOR run to 1e-13 of max |b|, beside the shared assembly of the same case. Checked here, on the CPU: the SOR solution
satisfies the shared system, and the oracle's Chorin step (the shared path, restated) reproduces EXPLICIT's pressure
and projected velocities.
"""
import numpy as np
import pytest

from conftest import explicit_golden_names, load_golden
from oracle import cpu

NAMES = explicit_golden_names()


def test_fixtures_exist():
    assert len(NAMES) >= 2


@pytest.mark.parametrize("name", NAMES)
def test_sor_solution_solves_the_shared_system(name):
    case, meta, z = load_golden(name)
    assert meta["rel_res"] <= 1e-12
    assert meta["max_div"] <= 1e-9


@pytest.mark.parametrize("name", NAMES)
def test_oracle_chorin_step_reproduces_explicit(name):
    case, meta, z = load_golden(name)
    g = case.grid
    o = cpu.solve_projection(g, z["types"], z["u"], z["v"], z["w"], z["p_in"], meta["rho"], meta["dt"],
                             meta["needs_compat"], 1e-13)
    assert o.asm.n == meta["n"]
    assert np.array_equal(o.asm.idp, z["idp"])
    x, xr = o.x, z["x"]
    if meta["singular"]:
        x, xr = x - x.mean(), xr - xr.mean()
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) <= 1e-9
    scale = max(np.abs(z["u"]).max(), np.abs(z["v"]).max())
    assert np.abs(o.u - z["u_out"]).max() <= 1e-9 * scale
    assert np.abs(o.v - z["v_out"]).max() <= 1e-9 * scale


def test_interior_air_is_outside_the_equivalence():
    """With EMPTY cells inside the grid (a free surface), EXPLICIT's coefficient toward them is 2 and the shared
    system's ring factor 1 (interior Dirichlet cells are not ring cells): the two pressures differ, so the routing
    holds only where every EMPTY and PRESSURE cell lies on the ring (tests/golden/limit_explicit_tank_2d_24.npz)."""
    case, meta, z = load_golden("limit_explicit_tank_2d_24")
    g = case.grid
    t = z["types"].reshape(g.Ny, g.Nx)
    assert (t[1:-1, 1:-1] == 2).any()  # EMPTY inside
    assert meta["rel_res"] > 1e-2  # EXPLICIT's pressure does not solve the shared system
    o = cpu.solve_projection(g, z["types"], z["u"], z["v"], z["w"], z["p_in"], meta["rho"], meta["dt"],
                             meta["needs_compat"], 1e-13)
    assert np.linalg.norm(o.x - z["x"]) / np.linalg.norm(z["x"]) > 1e-2


@pytest.mark.parametrize("name", NAMES)
def test_compatibility_on_changes_nothing_unless_singular(name):
    """The routing passes needsCompat = true: the compatibility step and the levelling act only on a singular system
    (PressureSolver3D.cpp:300-307, 181-211), which is when EXPLICIT removes its mean, so the flag leaves a
    non-singular step as it was."""
    case, meta, z = load_golden(name)
    args = (case.grid, z["types"], z["u"], z["v"], z["w"], z["p_in"], meta["rho"], meta["dt"])
    on = cpu.solve_projection(*args, True, 1e-13)
    off = cpu.solve_projection(*args, meta["needs_compat"], 1e-13)
    if not meta["singular"]:
        assert np.array_equal(on.x, off.x) and np.array_equal(on.u, off.u)
    x, xr = on.x - on.x.mean(), z["x"] - z["x"].mean()
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) <= 1e-9
