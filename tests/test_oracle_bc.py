"""The boundary-condition replay (MAC::EnforceVelocityBC and EnforcePressureBC, src/MAC.cpp:811-865): the oracle's
restatement, run on the lists the reference's own MAC::BuildBoundaryLists made (tests/golden/bc_*.npz), reproduces
the reference's fields bit for bit. The lists cover every kind a scene gives: no-slip, slip and sliding walls, a
space- and time-dependent inlet, the continuity outflow (with ApplyOutflowFlux), pressure outlets with and without a
prescribed p, interior solids, 2D and 3D."""
import numpy as np
import pytest

from conftest import bc_golden_names, load_golden
from oracle import cpu

NAMES = bc_golden_names()


def test_fixtures_exist():
    assert len(NAMES) >= 5


@pytest.mark.parametrize("name", NAMES)
def test_oracle_replay_bit_exact(name):
    case, meta, z = load_golden(name)
    u, v, w, p = cpu.bc_replay(z, z["u_in"], z["v_in"], z["w_in"], z["p_in"])
    assert np.array_equal(u, z["u_out"])
    assert np.array_equal(v, z["v_out"])
    assert np.array_equal(w, z["w_out"])
    assert np.array_equal(p, z["p_out"])


@pytest.mark.parametrize("name", NAMES)
def test_the_replay_changes_the_boundary(name):
    case, meta, z = load_golden(name)
    assert (z["u_out"] != z["u_in"]).any() and (z["p_out"] != z["p_in"]).any()


def test_every_kind_is_covered():
    kinds = set()
    outflow = copies_chain = 0
    for name in NAMES:
        case, meta, z = load_golden(name)
        kinds |= set(np.unique(z["ring_kind"]).tolist())
        outflow += len(z["outflow_comp"])
        # a copy that reads a value an earlier copy of the same field wrote (edges from faces, corners from edges)
        written = set()
        for c, d, s in zip(z["copy_comp"], z["copy_dst"], z["copy_src"]):
            copies_chain += (int(c), int(s)) in written
            written.add((int(c), int(d)))
    assert kinds == {0, 1, 2}
    assert outflow > 0 and copies_chain > 0
