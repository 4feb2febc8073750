"""FLIP's re-labelling from particles (FLIP3D::UpdateFluidCells, src/Methods/FLIP/FLIP3D.cpp:784-833; FLIP2D,
src/Methods/FLIP/FLIP2D.cpp:648-691; MAC::ResetFluidCells, src/MAC.cpp:556-589): the oracle against what the
reference's own code computed (tests/golden/flip_relabel_*.npz), then the Chorin step on the new labels."""
import numpy as np
import pytest

from conftest import flip_golden_names, load_golden
from nereus_cfd_b200 import workloads as W
from oracle import cpu

NAMES = flip_golden_names()


def test_fixtures_exist():
    assert len(NAMES) >= 2


def _origin(case):
    return [ax.face[0] for ax in case.grid.axes]


@pytest.mark.parametrize("name", NAMES)
def test_origin_is_the_first_ring_face(name):
    case, meta, z = load_golden(name)
    o = _origin(case)
    assert o[0] == meta["origin"][0] and o[1] == meta["origin"][1]
    if case.grid.dim == 3:
        assert o[2] == meta["origin"][2]


@pytest.mark.parametrize("name", NAMES)
def test_input_labels_are_the_scene_labels(name):
    case, meta, z = load_golden(name)
    assert np.array_equal(cpu.label_cells(case.grid, case.scene), z["types_in"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_relabel_bit_exact(name):
    case, meta, z = load_golden(name)
    out, skipped = cpu.update_fluid_cells(case.grid, z["types_in"], z["xyz"], meta["origin"], meta["dh"])
    assert skipped == 0
    assert np.array_equal(out, z["types"])
    assert not np.array_equal(out, z["types_in"])


@pytest.mark.parametrize("name", NAMES)
def test_particles_regenerate_from_the_seed(name):
    case, meta, z = load_golden(name)
    xyz = W.flip_particles(case, z["types_in"], meta["particle_seed"], meta["ppc"])
    assert np.array_equal(xyz, z["xyz"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_chorin_step_on_new_labels(name):
    case, meta, z = load_golden(name)
    o = cpu.solve_projection(case.grid, z["types"], z["u"], z["v"], z["w"], z["p_in"], meta["rho"], meta["dt"],
                             meta["needs_compat"], meta["tol"])
    assert o.asm.n == meta["n"]
    assert np.array_equal(o.asm.idp, z["idp"])
    assert np.linalg.norm(o.x - z["x"]) <= 1e-8 * np.linalg.norm(z["x"])


def test_in_place_order_matters():
    """The hole-filling pass reads its (i-1), (j-1), (k-1) neighbours after their own visit: a run of empty cells
    along +k inside the liquid fills completely, while the same run read only from the labels before the pass
    (a parallel, order-free rule) would fill its two end cells only."""
    case = W.flip_tank_3d(n=10, seed=3, a=0.95, b=0.95)
    g = case.grid
    t = np.full(g.shape, W.SOLID, dtype=np.uint8)
    t[1:-1, 1:-1, 1:-1] = W.EMPTY
    dh = g.dh
    org = _origin(case)
    fluid = [(i, j, k) for i in range(2, 8) for j in range(2, 8) for k in range(2, 8)
             if not (i == 4 and j == 4 and 3 <= k <= 6)]
    xyz = np.array([[org[0] + (j + 0.5) * dh, org[1] + (i + 0.5) * dh, org[2] + (k + 0.5) * dh]
                    for i, j, k in fluid])
    out, skipped = cpu.update_fluid_cells(g, t.reshape(-1), xyz, org)
    out = out.reshape(g.shape)
    assert skipped == 0
    assert all(out[4, 4, k] == W.FLUID for k in range(3, 7))


def test_particles_far_below_the_grid_are_skipped():
    case = W.flip_tank_2d(n=8)
    g = case.grid
    t = cpu.label_cells(g, case.scene)
    org = _origin(case)
    dh = g.dh
    xyz = np.array([[org[0] - 1.5 * dh, org[1] + 3.5 * dh, 0.0],      # more than a cell below in x: skipped
                    [org[0] + 3.5 * dh, org[1] - 0.5 * dh, 0.0],      # within one cell below in y: row 0
                    [np.nan, org[1] + 3.5 * dh, 0.0],                 # not finite: skipped
                    [org[0] + 3.5 * dh, np.inf, 0.0]])                # +inf: the top row
    out, skipped = cpu.update_fluid_cells(g, t, xyz, org)
    assert skipped == 2
