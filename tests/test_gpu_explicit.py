"""The EXPLICIT method's pressure and projection steps routed through the B200 backend: nereus_b200_project on the
EXPLICIT case (uniform 2D, compatibility on for a closed domain, where EXPLICIT removes the mean) reproduces what the
reference's own Explicit2D::Pressure (SOR to 1e-13 of max |b|) and ::Projection computed
(tests/golden/explicit_*.npz; src/Methods/Explicit/Explicit2D.cpp:48-120), to the parity bar of the other solves:
the mean-free pressure within 1e-6 relative L2, the projected velocities within 1e-6 of the largest input velocity.
"""
import numpy as np
import pytest

from conftest import explicit_golden_names, load_golden
from nereus_cfd_b200 import capi
from nereus_cfd_b200.pressure import MACGrid, PressureSolver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("name", explicit_golden_names())
def test_project_reproduces_explicit_step(nb, name, precision):
    case, meta, z = load_golden(name)
    g = case.grid
    m = MACGrid(g, z["types"].copy(), z["u"].copy(), z["v"].copy(), z["w"].copy(), z["p_in"].copy(), meta["rho"],
                meta["dt"])
    s = PressureSolver(precision)
    r = s.SolvePressure(m, tol=1e-10, needs_compat=meta["needs_compat"])
    s.DestroyPressureSolver()
    assert r.status == capi.NB_OK and r.rel_res <= 1e-10
    assert r.n == meta["n"] and bool(r.singular) == meta["singular"]
    idp = z["idp"]
    x = m.p[idp >= 0][np.argsort(idp[idp >= 0])]
    xr = z["x"]
    if meta["singular"]:
        x, xr = x - x.mean(), xr - xr.mean()
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) <= 1e-6
    scale = max(np.abs(z["u"]).max(), np.abs(z["v"]).max())
    assert np.abs(m.u - z["u_out"]).max() <= 1e-6 * scale
    assert np.abs(m.v - z["v_out"]).max() <= 1e-6 * scale
