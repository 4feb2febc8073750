"""Coarsening with x groups on stretched 3D grids (x_groups = 1, the default).

The stretched cylinder's x widths run from 0.0013 in its band to 0.066 at its ends against 0.0032 in y and z. Halving
every axis leaves coarse cells up to 20 times longer in x than across, where red-black point smoothing stalls; keeping
the wide x cells whole (and pairing the thin ones) keeps the coarse cells near cubes. Each solve below must meet its
tolerance with the reference's FP64 residual; the grouped hierarchy must need far fewer CG iterations than the halved
one, in both precisions and every FP32 kernel family. Solved to 1e-11 the two hierarchies' pressures agree within
1e-5. At 1e-8 the mixed solves lie further apart (measured against the reference's 1e-12 solve: 4.7e-4 grouped,
1.7e-5 halved; the FP64 ones 6.9e-8 and 3.9e-7): the cylinder's operator is ill-conditioned, so a relative residual
of 1e-8 bounds the pressure's error only loosely, and how much error the residual leaves in the smooth modes depends
on the Krylov space that made it (two short FP32 passes in the mixed form, one FP64 space in the plain one).
"""
import os

import numpy as np
import pytest

from nereus_cfd_b200 import capi, workloads as W
from nereus_cfd_b200.pressure import MACGrid, PressureSolver

pytestmark = pytest.mark.gpu


def solve(case, types, u, v, w, precision, tol, **opts):
    g = case.grid
    m = MACGrid(g, types.copy(), u.copy(), v.copy(), w.copy(), np.zeros(g.cells), case.rho, case.dt)
    s = PressureSolver(precision, **opts)
    r = s.SolvePressure(m, tol=tol, needs_compat=case.needs_compat)
    s.DestroyPressureSolver()
    return r, m


@pytest.fixture(scope="module")
def cylinder():
    case = W.stretched_cylinder_3d(192, 128, 128, seed=3)
    types = capi.label_cells(case.grid, case.scene)
    u, v, w = W.face_velocities(case.grid, types, case.seed, case.velocity_rule, case.fp32_velocity)
    return case, types, u, v, w


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_groups_cut_iterations_on_the_cylinder(nb, cylinder, precision):
    case, types, u, v, w = cylinder
    tol = 1e-8
    rg, mg = solve(case, types, u, v, w, precision, tol)
    rh, mh = solve(case, types, u, v, w, precision, tol, x_groups=0)
    for r in (rg, rh):
        assert r.status == capi.NB_OK and r.rel_res <= tol, r.as_dict()
    # measured on a B200: 16 against 74 (mixed), 16 against 73 (fp64)
    assert rg.iters_inner <= 20, rg.as_dict()
    assert rh.iters_inner >= 2 * rg.iters_inner, (rg.as_dict(), rh.as_dict())
    assert rg.max_div <= 10.0 * rh.max_div + 1e-12
    tight = 1e-11
    rg, mg = solve(case, types, u, v, w, precision, tight)
    rh, mh = solve(case, types, u, v, w, precision, tight, x_groups=0)
    for r in (rg, rh):
        assert r.status == capi.NB_OK and r.rel_res <= tight, r.as_dict()
    fluid = types.reshape(-1) == W.FLUID
    pg, ph = mg.p.reshape(-1)[fluid], mh.p.reshape(-1)[fluid]
    assert np.linalg.norm(pg - ph) / np.linalg.norm(ph) <= 1e-5


@pytest.mark.parametrize("family", [0, 1])
def test_groups_in_every_fp32_family(nb, cylinder, family):
    """pair_kernels 0 (per-cell transfers, k_restrict_x / k_prolong_x) and 1 (cell pairs): the colour-split layout
    is not used on stretched grids, so these two are the FP32 paths the grouped transfers run in."""
    case, types, u, v, w = cylinder
    tol = 1e-8
    r, m = solve(case, types, u, v, w, "mixed", tol, pair_kernels=family)
    assert r.status == capi.NB_OK and r.rel_res <= tol, r.as_dict()
    assert r.iters_inner <= 20, r.as_dict()
    tight = 1e-11
    r, m = solve(case, types, u, v, w, "mixed", tight, pair_kernels=family)
    ref, mref = solve(case, types, u, v, w, "mixed", tight)
    assert r.rel_res <= tight and ref.rel_res <= tight
    fluid = types.reshape(-1) == W.FLUID
    a, b = m.p.reshape(-1)[fluid], mref.p.reshape(-1)[fluid]
    assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5


def test_groups_on_a_graded_tank(nb):
    """A serving-trace-like grid: a 96^3 tank whose x widths grow by 1.04 over the outer cells of each side; the
    grouped hierarchy meets the tolerance, repeats its bits, and needs no more iterations than the halved one."""
    n = 96
    wx = W.band_stretched_widths(n, 1.0, 32, 0.5, 1.04)
    g = W.stretched_grid(3, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), [wx, np.full(n, 1.0 / n), np.full(n, 1.0 / n)])
    case = W.Case("graded_tank_96", g, W.walls_scene(3, outlet_face=1, inlet_face=0), 11)
    types = capi.label_cells(g, case.scene)
    u, v, w = W.face_velocities(g, types, case.seed, case.velocity_rule, case.fp32_velocity)
    r1, m1 = solve(case, types, u, v, w, "mixed", 1e-8)
    r2, m2 = solve(case, types, u, v, w, "mixed", 1e-8)
    r0, _ = solve(case, types, u, v, w, "mixed", 1e-8, x_groups=0)
    assert r1.status == capi.NB_OK and r1.rel_res <= 1e-8
    assert (r1.iters_inner, r1.rel_res) == (r2.iters_inner, r2.rel_res)
    assert np.array_equal(m1.p, m2.p)
    assert r1.iters_inner <= r0.iters_inner


@pytest.fixture(scope="module")
def reference(cylinder):
    """The reference's own solves of the cylinder (oracle/_ref/ref_harness: AMGCL SA+SPAI0 CG, run on this host, the
    way tests/suite_pressure.cpp:104-141 drives it) to 1e-12 and to 1e-8."""
    from oracle import refcase

    if not refcase.available():
        pytest.skip("oracle/_ref/ref_harness is not built")
    case, types, u, v, w = cylinder
    threads = os.cpu_count() or 1
    run = lambda tol: refcase.run(case, u, v, w, label_mode=1, types=types, solver=refcase.SOLVER_AMG, tol=tol,
                                  threads=threads, timeout=1800, lean=True)
    return run(1e-12), run(1e-8)


def test_cylinder_against_reference(nb, cylinder, reference):
    """The full 192x128x128 cylinder against the reference's solve at 1e-12 (the reference's own 1e-8 solve lies
    5.3e-8 from it, measured):
    - plain FP64 to 1e-8: pressure within 1e-6 relative L2 on the fluid cells (measured 6.9e-8);
    - mixed to 1e-8: the residual bar holds, but its pressure lies 4.7e-4 from the reference's (measured): two
      refinement passes of 8 FP32 CG iterations leave the smooth modes' error that one FP64 Krylov space of 16
      iterations removes, so the bar is 1e-3 here and 1e-6 only from a solve to 1e-11 (measured 1.4e-6 at 1e-10);
    - max |div u| within 10x of the reference's own at 1e-8 for both."""
    case, types, u, v, w = cylinder
    r12, r8 = reference
    assert r12.rel_res <= 1e-11 and r8.rel_res <= 1e-8
    fluid = types.reshape(-1) == W.FLUID
    ref = r12.p.reshape(-1)[fluid]
    err = lambda m: float(np.linalg.norm(m.p.reshape(-1)[fluid] - ref) / np.linalg.norm(ref))
    for precision, tol, bar in (("fp64", 1e-8, 1e-6), ("mixed", 1e-8, 1e-3), ("mixed", 1e-11, 1e-6)):
        r, m = solve(case, types, u, v, w, precision, tol)
        assert r.status == capi.NB_OK and r.rel_res <= tol, r.as_dict()
        assert r.n == r12.n and r.singular == int(r12.singular)
        assert err(m) <= bar, (precision, tol, err(m))
        assert r.max_div <= 10.0 * r8.max_div, (r.max_div, r8.max_div)
