"""A context reused across layouts gives what a fresh context gives, through the C ABI: a uniform grid of the same
sizes at another cell width (the hierarchy keeps its shape and captured iterations; the spacing tables and the
matrix scale are replaced) and a 2D grid after it, in both precisions, bit for bit."""
import copy

import numpy as np
import pytest

from nereus_cfd_b200 import serving, workloads as W
from nereus_cfd_b200.pressure import PressureSolver

pytestmark = pytest.mark.gpu


def sphere_box(L, n, seed):
    g = W.uniform_grid(3, (0.0, L, 0.0, L, 0.0, L), n)
    sph = W.Region(W.REGION_SOLID, W.PRIM_SPHERE, (0.5 * L, 0.5 * L, 0.5 * L), radius=0.15 * L)
    return W.Case("sphere_box_%g_%d" % (L, n), g, W.walls_scene(3, outlet_face=1, regions=[sph]), seed)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_rescaled_uniform_layout_equals_fresh(nb, precision):
    jobs = [serving.job_from_case(sphere_box(L, 24, s), tol=1e-9) for L, s in ((1.0, 5), (2.5, 6), (0.3, 7))]
    jobs.append(serving.job_from_case(W.closed_box_2d(40, seed=8), tol=1e-9))
    reused = PressureSolver(precision)
    for j in jobs:
        a, b = copy.deepcopy(j), copy.deepcopy(j)
        ra = reused.SolvePressure(a.grid, tol=j.tol, needs_compat=j.needs_compat)
        fresh = PressureSolver(precision)
        rb = fresh.SolvePressure(b.grid, tol=j.tol, needs_compat=j.needs_compat)
        fresh.DestroyPressureSolver()
        assert ra.status == rb.status == 0 and ra.rel_res <= j.tol
        assert (ra.iters_inner, ra.iters_outer, ra.rel_res) == (rb.iters_inner, rb.iters_outer, rb.rel_res)
        for f in ("p", "u", "v", "w"):
            assert np.array_equal(getattr(a.grid, f), getattr(b.grid, f)), f
    reused.DestroyPressureSolver()
