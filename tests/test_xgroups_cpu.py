"""The x-group planner of stretched coarsening (nereus_b200_x_groups, host only) against its rule restated here:
left to right, two interior x cells form one coarse cell when together they are at most three times the thinnest
y/z width (1.5 coarse y/z cells), else the cell stays whole."""
import numpy as np
import pytest

from nereus_cfd_b200 import capi, workloads as W


def plan(widths, yz):
    lib = capi.load()
    w = np.ascontiguousarray(widths, dtype=np.float64)
    out = np.zeros(len(w), dtype=np.int32)
    m = lib.nereus_b200_x_groups(w.ctypes.data_as(capi._dp), len(w), float(yz), out.ctypes.data_as(capi._ip))
    assert m > 0
    return out[:m].tolist()


def restated(widths, yz):
    out, j = [], 0
    while j < len(widths):
        two = j + 1 < len(widths) and widths[j] + widths[j + 1] <= 3.0 * yz
        out.append(2 if two else 1)
        j += 2 if two else 1
    return out


def test_cylinder_groups():
    case = W.stretched_cylinder_3d(192, 128, 128)
    wx = case.grid.interior_widths[0]
    got = plan(wx, 0.41 / 128)
    assert got == restated(wx, 0.41 / 128)
    assert sum(got) == 192 and len(got) == 148
    # the thin band and its neighbours are paired, the wide ends stay whole
    assert got[0] == 1 and got[-1] == 1 and 2 in got


@pytest.mark.parametrize("seed", range(5))
def test_random_widths(seed):
    rng = np.random.default_rng(seed)
    wx = rng.uniform(0.2, 3.0, size=int(rng.integers(1, 300)))
    got = plan(wx, 1.0)
    assert got == restated(wx, 1.0)
    assert sum(got) == len(wx)


def test_uniform_thin_cells_pair_everywhere():
    assert plan(np.full(10, 0.5), 1.0) == [2] * 5
    assert plan(np.full(7, 0.5), 1.0) == [2, 2, 2, 1]
    assert plan(np.full(4, 2.0), 1.0) == [1] * 4


def test_bad_input():
    lib = capi.load()
    w = np.ones(4)
    out = np.zeros(4, dtype=np.int32)
    assert lib.nereus_b200_x_groups(w.ctypes.data_as(capi._dp), 0, 1.0, out.ctypes.data_as(capi._ip)) == \
        capi.NB_BAD_INPUT
    assert lib.nereus_b200_x_groups(w.ctypes.data_as(capi._dp), 4, 0.0, out.ctypes.data_as(capi._ip)) == \
        capi.NB_BAD_INPUT
