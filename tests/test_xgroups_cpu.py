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


def maps(widths, yz):
    lib = capi.load()
    w = np.ascontiguousarray(widths, dtype=np.float64)
    n = len(w)
    xp = np.zeros(n + 2, dtype=np.int32)
    xr = np.zeros(n + 2, dtype=np.int32)
    nc = lib.nereus_b200_x_maps(w.ctypes.data_as(capi._dp), n, float(yz), xp.ctypes.data_as(capi._ip),
                                xr.ctypes.data_as(capi._ip))
    assert nc >= 0
    return nc, xp, xr[:nc]


def prolongation_1d(xp, nc):
    """P along x as the prolongation kernels read xp: a fine cell gives its parent 1 (one child) or 3/4, and the
    other contributor 1/4."""
    P = np.zeros((len(xp), nc))
    for j, x in enumerate(xp):
        parent, other, single = x & 0x7FFF, (x >> 15) & 0x7FFF, (x >> 30) & 1
        if single:
            assert other == parent
            P[j, parent] += 1.0
        else:
            assert abs(other - parent) == 1
            P[j, parent] += 0.75
            P[j, other] += 0.25
    return P


def restriction_taps_1d(xr, nf):
    """R along x as the restriction kernels read xr (the taps of XrTaps), rows for the interior coarse cells."""
    R = np.zeros((len(xr), nf))
    for J in range(1, len(xr) - 1):
        x = int(xr[J])
        f0, two, before, after = x & 0x7FFF, (x >> 15) & 1, (x >> 16) & 1, (x >> 17) & 1
        if before:
            R[J, f0 - 1] += 0.25
        R[J, f0] += 0.75 if two else 1.0
        if two:
            R[J, f0 + 1] += 0.75
        if after:
            R[J, f0 + (2 if two else 1)] += 0.25
    return R


@pytest.mark.parametrize("case", ["cylinder", "random0", "random1", "random2"])
def test_maps_restrict_with_the_transpose(case):
    """The restriction taps are the transpose of the prolongation weights on every interior coarse cell, each fine
    interior cell has exactly one parent whose children include it, and the groups are the planner's."""
    if case == "cylinder":
        wx, yz = W.stretched_cylinder_3d(192, 128, 128).grid.interior_widths[0], 0.41 / 128
    else:
        rng = np.random.default_rng(int(case[-1]))
        wx, yz = rng.uniform(0.3, 2.5, size=int(rng.integers(8, 200))), 1.0
    nc, xp, xr = maps(wx, yz)
    counts = plan(wx, yz)
    if nc == 0:
        assert all(c == 2 for c in counts[:-1])
        return
    assert nc == len(counts) + 2
    nf = len(wx) + 2
    P = prolongation_1d(xp, nc)
    R = restriction_taps_1d(xr, nf)
    assert np.array_equal(R[1:nc - 1], P.T[1:nc - 1])
    # children: xr's children of J are exactly the fine cells whose parent is J
    for J in range(1, nc - 1):
        f0, two = int(xr[J]) & 0x7FFF, (int(xr[J]) >> 15) & 1
        kids = [f0, f0 + 1] if two else [f0]
        assert [j for j in range(nf) if (int(xp[j]) & 0x7FFF) == J] == kids
        assert len(kids) == counts[J - 1]
    # the rings map onto the rings
    assert int(xp[0]) & 0x7FFF == 0 and int(xp[-1]) & 0x7FFF == nc - 1


def test_maps_regular_pairing_is_left_to_the_plain_kernels():
    nc, _, _ = maps(np.full(12, 0.5), 1.0)
    assert nc == 0
