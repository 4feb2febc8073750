"""A CPU model of the concurrency argument behind k_relabel_fill and k_relabel_settle (nereus_cfd_b200/csrc/
nb_relabel.cu). It models the kernels' algorithm; the kernels themselves are tested against the reference in
test_gpu_flip.py.

The hole pass of FLIP's UpdateFluidCells (src/Methods/FLIP/FLIP3D.cpp:809-832) is serial and in place. On the device
every interior cell is evaluated by its own thread in any order, filled cells are marked, a fill follows its chain
upward, and the cells that may still be filled go on a list that one block then settles with fresh reads. Here any
read of a cell filled by another thread may return its value from before the fill, as a read from a non-coherent L1
may. With each lower neighbour read once for both the count and the "may still be filled" figure, the result is the
serial pass's in every run; with two reads, as the kernel once had, a cell can fall out of both.
"""
import numpy as np
import pytest

from nereus_cfd_b200 import workloads as W
from oracle import cpu

FILLED = 0x80


def _marked(g, t, xyz, origin):
    """Reset and particle marking (the oracle's first two steps), without the hole pass."""
    out, _ = cpu.update_fluid_cells(g, t, np.zeros((0, 3)), origin)
    nz = g.Nz if g.dim == 3 else 1
    for x, y, z in xyz:
        idx = []
        for v, o, N in ((y, origin[1], g.Ny), (x, origin[0], g.Nx), (z, origin[2], nz)):
            q = (v - o) / g.dh
            idx.append(-1 if not q > -1 else (N - 1 if q >= N else int(q)))
        if g.dim == 2:
            idx[2] = 0
        if min(idx) < 0:
            continue
        c = (idx[0] * g.Nx + idx[1]) * nz + idx[2]
        if out[c] == W.EMPTY:
            out[c] = W.FLUID
    return out


def _device_pass(g, marked, rng, reads_once, p_stale=0.5):
    dim, Nx, Ny = g.dim, g.Nx, g.Ny
    nz = g.Nz if dim == 3 else 1
    t = marked.astype(np.int64).copy()
    sI, sJ, thr = Nx * nz, (nz if dim == 3 else 1), 2 * dim - 1
    lower = [sI, 1, sJ] if dim == 3 else [sI, 1]

    def rd(c, fresh=False):
        v = int(t[c])
        return W.EMPTY if (not fresh and v == FILLED and rng.random() < p_stale) else v

    def count(c, fresh=False):
        return (sum(int(rd(c + s, fresh) == W.FLUID) for s in lower) +
                sum(int(rd(c - s, fresh) in (W.FLUID, FILLED)) for s in lower))

    def coords(c):
        i, r = divmod(c, sI)
        return (i,) + (divmod(r, sJ) if dim == 3 else (0, r))

    def chase(c, i, j, m, fresh=False):
        last = nz - 2 if dim == 3 else Nx - 2
        while True:
            u = -1
            if m < last and rd(c + 1, fresh) == W.EMPTY:
                u, m = c + 1, m + 1
            elif dim == 3 and j < Nx - 2 and rd(c + sJ, fresh) == W.EMPTY:
                u, j = c + sJ, j + 1
            elif i < Ny - 2 and rd(c + sI, fresh) == W.EMPTY:
                u, i = c + sI, i + 1
            if u < 0 or count(u, fresh) < thr:
                return
            t[u] = FILLED
            c = u

    cells = [(i, j, m) for i in range(1, Ny - 1) for j in (range(1, Nx - 1) if dim == 3 else [0])
             for m in range(1, (nz - 1) if dim == 3 else (Nx - 1))]
    rng.shuffle(cells)
    pending = []
    for i, j, m in cells:
        c = (i * Nx + j) * nz + m if dim == 3 else i * Nx + m
        if int(t[c]) != W.EMPTY:
            continue
        interior = [i > 1, m > 1, j > 1][:len(lower)]
        if reads_once:
            vals = [rd(c - s) for s in lower]
            f = sum(int(rd(c + s) == W.FLUID) for s in lower) + sum(int(v in (W.FLUID, FILLED)) for v in vals)
            maybe = sum(int(ok and v == W.EMPTY) for ok, v in zip(interior, vals))
        else:
            f = count(c)
            maybe = sum(int(ok and rd(c - s) == W.EMPTY) for ok, s in zip(interior, lower))
        if f >= thr:
            t[c] = FILLED
            chase(c, i, j, m)
        elif f + maybe >= thr:
            pending.append(c)
    while True:  # the settling block: fresh reads after each barrier
        changed = False
        for c in pending:
            if int(t[c]) == W.EMPTY and count(c, True) >= thr:
                t[c] = FILLED
                chase(c, *coords(c), fresh=True)
                changed = True
        if not changed:
            break
    t[t == FILLED] = W.FLUID
    return t.astype(np.uint8)


@pytest.mark.parametrize("builder,kwargs", [(W.flip_tank_3d, {"n": 10, "seed": 1}),
                                            (W.flip_tank_2d, {"n": 20, "seed": 2})])
def test_one_read_per_neighbour_gives_the_serial_result(builder, kwargs):
    case = builder(**kwargs)
    g = case.grid
    t0 = cpu.label_cells(g, case.scene)
    origin = [ax.face[0] for ax in g.axes]
    rng = np.random.default_rng(11)
    for holes in (0.3, 0.6, 0.8):
        for seed in range(3):
            xyz = W.flip_particles(case, t0, 7 + seed, 2, hole_fraction=holes)
            ref, _ = cpu.update_fluid_cells(g, t0, xyz, origin)
            marked = _marked(g, t0, xyz, origin)
            for _ in range(2):
                assert np.array_equal(_device_pass(g, marked, rng, reads_once=True), ref)
