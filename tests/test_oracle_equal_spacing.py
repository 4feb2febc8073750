"""The reference's own separator between "a branch is wrong" and "the stretching is wrong"
(tests/suite_exact3d.cpp:219-231, 368-382): the rectilinear branch (finite-volume coefficients A_f/d_f, RHS weighted
by the cell volume, scale 1) at EQUAL spacing must reproduce the uniform branch (coefficient 1, scale 1/dh^2). The
two solve the same system scaled differently, so they agree to the solver's tolerance: the reference asserts the
velocity to 1e-11 relative and the pressure to 1e-10 absolute. Checked here on the oracle's two branches."""
import numpy as np
import pytest

from nereus_cfd_b200 import workloads as W
from oracle import cpu


def _equal_spacing_twin(case):
    g = case.grid
    n = [ax.n - 2 for ax in g.axes[:g.dim]]
    widths = [np.full(k, g.dh) for k in n]
    twin = W.stretched_grid(g.dim, g.domain, widths)
    return W.Case(case.name + "_equal_spacing", twin, case.scene, case.seed, case.rho, case.dt, case.needs_compat,
                  case.tol, case.velocity_rule, case.fp32_velocity, case.method)


@pytest.mark.parametrize("case", [W.sphere_outlet_3d(12, seed=51), W.closed_box_2d(16, seed=52),
                                  W.inflow_outflow_3d(8, seed=53)], ids=lambda c: c.name)
def test_rectilinear_branch_at_equal_spacing_reproduces_uniform(case):
    twin = _equal_spacing_twin(case)
    g, gt = case.grid, twin.grid
    assert not g.nonuniform and gt.nonuniform
    types = cpu.label_cells(g, case.scene)
    assert np.array_equal(cpu.label_cells(gt, twin.scene), types)
    u, v, w = W.face_velocities(g, types, case.seed, case.velocity_rule, case.fp32_velocity)
    a = cpu.solve_projection(g, types, u, v, w, np.zeros(g.cells), case.rho, case.dt, case.needs_compat, 1e-13)
    b = cpu.solve_projection(gt, types, u, v, w, np.zeros(g.cells), case.rho, case.dt, case.needs_compat, 1e-13)
    assert np.array_equal(a.asm.idp, b.asm.idp)
    scale = max(np.abs(u).max(), np.abs(v).max())
    for x, y in ((a.u, b.u), (a.v, b.v)) + (((a.w, b.w),) if g.dim == 3 else ()):
        assert np.abs(x - y).max() <= 1e-11 * scale
    pa, pb = a.x, b.x
    if a.asm.singular:
        pa, pb = pa - pa.mean(), pb - pb.mean()
    assert np.abs(pa - pb).max() <= 1e-10 * max(np.abs(pa).max(), 1.0)
