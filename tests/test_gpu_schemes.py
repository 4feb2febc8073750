"""The incremental scheme and the Chorin warm start on the B200 (nereus_b200_project_ex through the PressureSolver
mirror) against the fixtures the reference wrote for them.

Bars: the final pressure within 1e-6 relative L2 of the reference's (which solved to 1e-12; here 1e-10), the
prescribed ring values bit-exact, the velocity correction within 1e-6 of the reference's relative to its size,
max |div u| below 1e-6; the warm start needs fewer iterations than the same solve from zero.
"""
import numpy as np
import pytest

from conftest import load_golden, scheme_golden_names
from nereus_cfd_b200 import capi
from nereus_cfd_b200.pressure import MACGrid, PressureSolver

pytestmark = pytest.mark.gpu
NAMES = scheme_golden_names()


def grids(case, meta, z):
    g = case.grid
    cur = MACGrid(g, z["types"].copy(), z["u"].copy(), z["v"].copy(), z["w"].copy(), z["p_in"].copy(), meta["rho"],
                  meta["dt"])
    ant = MACGrid(g, z["types"].copy(), z["u"].copy(), z["v"].copy(), z["w"].copy(), z["p_prev"].copy(),
                  meta["rho"], meta["dt"])
    return cur, ant


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("name", NAMES)
def test_scheme_matches_reference(nb, name, precision):
    case, meta, z = load_golden(name)
    cur, ant = grids(case, meta, z)
    scheme = capi.SCHEME_INCREMENTAL if meta["scheme"] == 1 else capi.SCHEME_CHORIN
    s = PressureSolver(precision)
    s.InitializePressureSolver(cur, scheme, warm_start=meta["scheme"] == 2)
    r = s.SolvePressure(cur, tol=1e-10, needs_compat=meta["needs_compat"], grid_ant=ant)
    assert r.status == capi.NB_OK
    assert r.rel_res <= 1e-10
    final = z["p_final"]
    assert np.linalg.norm(cur.p - final) <= 1e-6 * np.linalg.norm(final)
    t = z["types"]
    assert np.array_equal(cur.p[t == 4], final[t == 4])
    for got, ref, inp in ((cur.u, z["u_out"], z["u"]), (cur.v, z["v_out"], z["v"]), (cur.w, z["w_out"], z["w"])):
        if ref.size:
            assert np.linalg.norm(got - ref) <= 1e-6 * max(np.linalg.norm(ref - inp), 1e-300)
    assert r.max_div < 1e-6
    if meta["scheme"] == 2:
        cold_grid, _ = grids(case, meta, z)
        c = PressureSolver(precision)
        c.InitializePressureSolver(cold_grid)
        rc = c.SolvePressure(cold_grid, tol=1e-10, needs_compat=meta["needs_compat"])
        assert r.iters_inner < rc.iters_inner
        c.DestroyPressureSolver()
    s.DestroyPressureSolver()


def test_incremental_needs_the_previous_step(nb):
    name = [n for n in NAMES if n.startswith("incremental_")][0]
    case, meta, z = load_golden(name)
    cur, _ = grids(case, meta, z)
    s = PressureSolver("mixed")
    s.InitializePressureSolver(cur, capi.SCHEME_INCREMENTAL)
    with pytest.raises(capi.NBError):
        s.SolvePressure(cur, grid_ant=None)
    # and through the C ABI directly: no p_prev
    g = case.grid
    st = nb.nereus_b200_project_ex(s.ctx, capi.ptr(cur.u), capi.ptr(cur.v), capi.ptr(cur.w), capi.ptr(cur.p), None,
                                   1.0, 1e-3, capi.SCHEME_INCREMENTAL, 0, 0, 1e-8, None)
    assert st == capi.NB_BAD_INPUT
    s.DestroyPressureSolver()
