"""Known answers the reference's FLIP suite holds for the pressure path (tests/suite_flip.cpp: a still tank stays
still; no flux through solids), on the oracle's projection."""
import numpy as np

from nereus_cfd_b200 import workloads as W
from oracle import cpu


def test_still_tank_stays_still():
    """Zero face velocities in a tank with air above (EMPTY, p = 0): b = 0, so p = 0 and nothing moves."""
    case = W.flip_tank_3d(12, seed=61)
    g = case.grid
    types = cpu.label_cells(g, case.scene)
    u, v, w = [np.zeros(int(np.prod(s))) for s in (g.u_shape(), g.v_shape(), g.w_shape())]
    o = cpu.solve_projection(g, types, u, v, w, np.zeros(g.cells), case.rho, case.dt, False, 1e-12)
    assert o.asm.n > 0
    assert not o.x.any() and not o.u.any() and not o.v.any() and not o.w.any()


def test_no_flux_through_solids():
    """After the projection, every face with a SOLID cell on either side keeps its zero (ProjectPressure skips wall
    faces, FaceGate, src/headers/Core/MAC.h:271-274)."""
    case = W.sphere_outlet_3d(12, seed=62)
    g = case.grid
    types = cpu.label_cells(g, case.scene)
    u, v, w = W.face_velocities(g, types, case.seed)
    o = cpu.solve_projection(g, types, u, v, w, np.zeros(g.cells), case.rho, case.dt, False, 1e-12)
    t = types.reshape(g.shape)
    for c, (f_in, f_out) in enumerate(((u, o.u), (v, o.v), (w, o.w))):
        shape = [g.u_shape(), g.v_shape(), g.w_shape()][c]
        ax = [1, 0, 2][c]
        pad = [(0, 0)] * 3
        pad[ax] = (1, 1)
        tp = np.pad(t, pad, constant_values=W.SOLID)
        lo, hi = [slice(None)] * 3, [slice(None)] * 3
        lo[ax], hi[ax] = slice(0, -1), slice(1, None)
        wall = ((tp[tuple(lo)] == W.SOLID) | (tp[tuple(hi)] == W.SOLID)).reshape(-1)
        assert wall.any()
        assert not f_out.reshape(shape).reshape(-1)[wall].any()
        assert (f_out != f_in).any()  # the projection did act elsewhere
