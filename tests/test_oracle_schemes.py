"""The oracle's restatement of the incremental scheme and the Chorin warm start against the fixtures the reference
itself wrote (tests/golden/incremental_*, warm_*: SolvePressure from gridAnt, then Project)."""
import numpy as np
import pytest

from conftest import load_golden, scheme_golden_names
from oracle import cpu

NAMES = scheme_golden_names()


def test_scheme_fixtures_present():
    assert any(n.startswith("incremental_") for n in NAMES)
    assert any(n.startswith("warm_") for n in NAMES)


def run(name):
    case, meta, z = load_golden(name)
    incremental = meta["scheme"] == 1
    r = cpu.solve_scheme(case.grid, z["types"], z["u"], z["v"], z["w"], z["p_in"], z["p_prev"], meta["rho"],
                         meta["dt"], meta["needs_compat"], meta["tol"], incremental, warm=meta["scheme"] == 2)
    return case, meta, z, r


@pytest.mark.parametrize("name", NAMES)
def test_rhs_bit_exact(name):
    case, meta, z, r = run(name)
    assert np.array_equal(r.b_raw, z["b_raw"])
    assert np.array_equal(r.b, z["b"])


@pytest.mark.parametrize("name", NAMES)
def test_solution_iterations_and_pressure(name):
    case, meta, z, r = run(name)
    assert r.iters == meta["iters"]
    if meta["scheme"] == 2:
        assert meta["iters"] < meta["cold_iters"]  # the guess is close to the answer
    xr = z["x"]
    if meta["singular"] and meta["scheme"] == 2:
        xr, xo = xr - xr.mean(), r.x - r.x.mean()
    else:
        xo = r.x
    assert np.linalg.norm(xo - xr) <= 1e-9 * np.linalg.norm(xr)
    final = z["p_final"]
    assert np.linalg.norm(r.p - final) <= 1e-9 * np.linalg.norm(final)
    t = z["types"]
    assert np.array_equal(r.p[t == 4], final[t == 4])  # the prescribed ring, put back exactly


@pytest.mark.parametrize("name", [n for n in NAMES if n.startswith("incremental_")])
def test_increment_ring_and_velocity(name):
    case, meta, z, r = run(name)
    t = z["types"]
    # after the solve the PRESSURE ring carries the increment p_b(t^{n+1}) - p_b(t^n)
    assert np.allclose(z["p"][t == 4], (z["p_in"] - z["p_prev"])[t == 4], rtol=0, atol=1e-15)
    # the projection of the reference's own increment reproduces its velocities exactly
    gv = cpu.GridView(case.grid, t)
    uu, vv = z["u"].copy(), z["v"].copy()
    ww = z["w"].copy() if z["w"].size else np.zeros(1)
    p = np.ascontiguousarray(z["p"])
    cpu.lib().or_project(gv.ref, cpu._p(uu, cpu._dp), cpu._p(vv, cpu._dp), cpu._p(ww, cpu._dp), cpu._p(p, cpu._dp),
                         meta["rho"], meta["dt"])
    assert np.array_equal(uu, z["u_out"])
    assert np.array_equal(vv, z["v_out"])
    if z["w"].size:
        assert np.array_equal(ww, z["w_out"])
