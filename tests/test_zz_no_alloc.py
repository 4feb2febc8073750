"""The allocation-free IDP numbering (nereus_b200_number_unknowns_noalloc) against the context path
(nereus_b200_set_layout + nereus_b200_get_idp / nereus_b200_system_size), through the C ABI.

IDP numbers are integers: the two paths must agree exactly, on two calls in a row (the second call reuses the
per-device scratch the first one left behind). The file is named to be collected last, and it passes on its own in a
fresh process as well.
"""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from nereus_cfd_b200 import capi, workloads as W
from nereus_cfd_b200.pressure import MACGrid, PressureSolver

pytestmark = pytest.mark.gpu
MAX_LINES = 262144  # NB_NOALLOC_MAX_LINES


def context_numbering(grid, types):
    s = PressureSolver("fp64")
    w = np.zeros(int(np.prod(grid.w_shape()))) if grid.dim == 3 else np.zeros(1)
    m = MACGrid(grid, np.ascontiguousarray(types, dtype=np.uint8).reshape(-1).copy(),
                np.zeros(int(np.prod(grid.u_shape()))), np.zeros(int(np.prod(grid.v_shape()))), w,
                np.zeros(grid.cells), 1.0, 1.0)
    s.InitializePressureSolver(m)
    idp, n = s.IDP(), s.SystemSize()
    s.DestroyPressureSolver()
    return idp, n


def noalloc_numbering(nb, grid, types, calls=2):
    import torch

    dev = torch.cuda.current_device()
    t = torch.from_numpy(np.ascontiguousarray(types, dtype=np.uint8).reshape(-1)).to("cuda")
    out = []
    for _ in range(calls):
        idp = torch.zeros(grid.cells, dtype=torch.int32, device="cuda")
        n = torch.full((1,), -7, dtype=torch.int32, device="cuda")
        st = nb.nereus_b200_number_unknowns_noalloc(dev, grid.dim, grid.Nx, grid.Ny, grid.Nz, t.data_ptr(),
                                                    idp.data_ptr(), n.data_ptr(),
                                                    torch.cuda.current_stream().cuda_stream)
        capi.check(st)
        torch.cuda.synchronize()
        out.append((idp.cpu().numpy(), int(n.item())))
    return out


@pytest.mark.parametrize("name", golden_names())
def test_matches_context_numbering(nb, name):
    case, meta, z = load_golden(name)
    ref_idp, ref_n = context_numbering(case.grid, z["types"])
    assert ref_n == meta["n"]
    for idp, n in noalloc_numbering(nb, case.grid, z["types"]):
        assert n == ref_n
        assert np.array_equal(idp, ref_idp)
        assert np.array_equal(idp, z["idp"].reshape(-1))


def random_layout(grid, seed):
    rng = np.random.default_rng(seed)
    return rng.choice(np.array([0, 0, 0, 1, 2, 4], dtype=np.uint8), size=grid.shape)


@pytest.mark.parametrize("dim", [2, 3])
def test_matches_at_the_line_limit(nb, dim):
    if dim == 3:  # (Ny-2)*(Nx-2) = 512*512 interior lines
        grid = W.stretched_grid(3, (0, 1, 0, 1, 0, 1), [np.full(512, 1 / 512), np.full(512, 1 / 512),
                                                        np.full(3, 1 / 3)])
    else:  # Ny-2 = 262144 interior rows of 3 cells
        grid = W.stretched_grid(2, (0, 1, 0, 1), [np.full(3, 1 / 3), np.full(MAX_LINES, 1 / MAX_LINES)])
    types = random_layout(grid, 11 + dim)
    ref_idp, ref_n = context_numbering(grid, types)
    assert ref_n > 0
    for idp, n in noalloc_numbering(nb, grid, types):
        assert n == ref_n
        assert np.array_equal(idp, ref_idp)


def test_sphere_then_tank_back_to_back(nb):
    # a changed layout on the next call: nothing of the first call's scratch may leak into the second
    a = W.sphere_outlet_3d(40)
    b = W.flip_tank_3d(40)
    ta, tb = capi.label_cells(a.grid, a.scene), capi.label_cells(b.grid, b.scene)
    ra, rb = context_numbering(a.grid, ta), context_numbering(b.grid, tb)
    (ia, na), = noalloc_numbering(nb, a.grid, ta, calls=1)
    (ib, nbb), = noalloc_numbering(nb, b.grid, tb, calls=1)
    assert na == ra[1] and np.array_equal(ia, ra[0])
    assert nbb == rb[1] and np.array_equal(ib, rb[0])


def test_beyond_the_limit_is_bad_input(nb):
    import torch

    Nx, Ny, Nz = 2 + 512, 2 + 513, 3  # 513*512 lines > the maximum
    t = torch.zeros(Nx * Ny * Nz, dtype=torch.uint8, device="cuda")
    idp = torch.zeros(Nx * Ny * Nz, dtype=torch.int32, device="cuda")
    n = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = nb.nereus_b200_number_unknowns_noalloc(torch.cuda.current_device(), 3, Nx, Ny, Nz, t.data_ptr(),
                                                idp.data_ptr(), n.data_ptr(), None)
    assert st == capi.NB_BAD_INPUT
    assert b"262144" in nb.nereus_b200_last_error()
    st = nb.nereus_b200_number_unknowns_noalloc(torch.cuda.current_device(), 3, Nx, Ny, Nz, None, None, None, None)
    assert st == capi.NB_BAD_INPUT
