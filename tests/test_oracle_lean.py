"""The reference harness's lean result (NB_REF_LEAN=1, used at the benchmark sizes) carries the same solution, pressure
and projected velocities as the full one, without the labels, numbering, matrix and right-hand sides."""
import numpy as np
import pytest

from nereus_cfd_b200 import workloads as W
from oracle import cpu, refcase


@pytest.mark.skipif(not refcase.available(), reason="oracle/_ref/ref_harness is not built")
@pytest.mark.parametrize("solver", [refcase.SOLVER_CG, refcase.SOLVER_AMG])
def test_lean_result_matches_full(solver):
    case = W.sphere_outlet_3d(10, seed=7)
    types = cpu.label_cells(case.grid, case.scene)
    u, v, w = W.face_velocities(case.grid, types, case.seed)
    full = refcase.run(case, u, v, w, label_mode=1, types=types, solver=solver, tol=1e-10)
    lean = refcase.run(case, u, v, w, label_mode=1, types=types, solver=solver, tol=1e-10, lean=True)
    assert full.val.size > 0 and lean.val.size == 0 and lean.types.size == 0 and lean.b.size == 0
    assert (lean.n, lean.iters, lean.singular) == (full.n, full.iters, full.singular)
    for a in ("x", "p", "u", "v", "w"):
        assert np.array_equal(getattr(lean, a), getattr(full, a)), a
    assert lean.rel_res == full.rel_res and lean.max_div == full.max_div
