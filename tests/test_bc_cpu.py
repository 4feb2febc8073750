"""The boundary-condition replay's C ABI on the CPU: nereus_b200_bc_create reads the reference's lists through
nb_bc_lists (the ctypes layout in capi.BcLists must match the C struct) and refuses a bad list before it looks for a
device: a component outside the grid's, an index outside its field, a ring kind other than 0, 1, 2, a null list."""
import ctypes

import numpy as np
import pytest

from conftest import bc_golden_names, cuda_ok, load_golden
from nereus_cfd_b200 import build, capi
from nereus_cfd_b200.boundary import BoundaryReplay

NAMES = bc_golden_names()


@pytest.fixture(scope="module")
def lib():
    build.build()
    return capi.load()


def _dims(case):
    g = case.grid
    return g.dim, g.Nx, g.Ny, (g.Nz if g.dim == 3 else 1)


def _create(lists, dims):
    try:
        BoundaryReplay(lists, *dims)
        return capi.NB_OK
    except capi.NBError as e:
        return e.status


@pytest.mark.parametrize("name", NAMES)
def test_valid_lists_reach_the_device_check(lib, name):
    case, meta, z = load_golden(name)
    st = _create(dict(z), _dims(case))
    assert st == (capi.NB_OK if cuda_ok() else capi.NB_NO_DEVICE)


def test_bad_lists_are_bad_input(lib):
    name = [n for n in NAMES if "_3d_" in n][0]
    case, meta, z = load_golden(name)
    dims = _dims(case)
    base = dict(z)

    def with_(key, fn):
        d = dict(base)
        d[key] = fn(np.array(base[key]).copy())
        return d

    big = lambda a: np.where(np.arange(len(a)) == 0, 10 ** 8, a)
    cases = [with_("presc_comp", lambda a: np.where(np.arange(len(a)) == 0, 3, a)),
             with_("presc_index", big), with_("copy_src", big), with_("copy_dst", lambda a: np.where(
                 np.arange(len(a)) == 0, -1, a)), with_("solid1", big), with_("ring_dst", big),
             with_("ring_kind", lambda a: np.where(np.arange(len(a)) == 0, 3, a))]
    if len(base["outflow_comp"]):
        cases.append(with_("outflow_outer", big))
    for d in cases:
        assert _create(d, dims) == capi.NB_BAD_INPUT
    # a 2D grid has no w
    name2 = [n for n in NAMES if "_2d_" in n][0]
    case2, _, z2 = load_golden(name2)
    d = dict(z2)
    d["presc_comp"] = np.full(len(z2["presc_comp"]), 2, dtype=np.int32)
    assert _create(d, _dims(case2)) == capi.NB_BAD_INPUT
    assert lib.nereus_b200_bc_create(0, None, None) == capi.NB_BAD_INPUT
    assert lib.nereus_b200_bc_enforce_velocity(None, None, None, None, None, None) == capi.NB_BAD_INPUT
    assert lib.nereus_b200_bc_enforce_pressure(None, None, None, None) == capi.NB_BAD_INPUT
    lib.nereus_b200_bc_destroy(None)
