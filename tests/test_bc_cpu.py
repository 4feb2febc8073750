"""The boundary-condition replay's C ABI on the CPU: nereus_b200_bc_create reads the reference's lists through
nb_bc_lists (the ctypes layout in capi.BcLists must match the C struct) and refuses a bad list before it looks for a
device: a component outside the grid's, an index outside its field, a ring kind other than 0, 1, 2, a null list."""
import ctypes

import numpy as np
import pytest

from conftest import bc_golden_names, cuda_ok, load_golden
from nereus_cfd_b200 import build, capi
from nereus_cfd_b200.boundary import BoundaryReplay
from oracle import cpu

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


def _run_levels(ops, levels, fields, values, null_zero):
    """Each level as one parallel scatter: every source of the level read before any destination is written."""
    comp, dst, src, val = ops
    for lv in range(int(levels.max()) + 1 if len(levels) else 0):
        sel = np.nonzero(levels == lv)[0]
        keys = set(zip(comp[sel].tolist(), dst[sel].tolist()))
        assert len(keys) == len(sel), "two writes of one destination in a level"
        reads = {(int(c), int(s)) for c, s in zip(comp[sel], src[sel]) if s >= 0}
        assert not (reads & keys), "a level reads a value it writes"
        new = []
        for q in sel:
            f = fields[comp[q]]
            if src[q] >= 0:
                new.append(f[src[q]])
            elif val[q] >= 0:
                new.append(values[val[q]] if values is not None else (0.0 if null_zero else None))
            else:
                new.append(0.0)
        for q, x in zip(sel, new):
            if x is not None:
                fields[comp[q]][dst[q]] = x


def _velocity_ops(z):
    comp, dst, src, val = [], [], [], []
    for c in range(3):
        n = len(z["solid%d" % c])
        comp += [c] * n; dst += list(z["solid%d" % c]); src += [-1] * n; val += [-1] * n
    n = len(z["presc_comp"])
    comp += list(z["presc_comp"]); dst += list(z["presc_index"]); src += [-1] * n; val += list(range(n))
    n = len(z["copy_comp"])
    comp += list(z["copy_comp"]); dst += list(z["copy_dst"]); src += list(z["copy_src"]); val += [-1] * n
    return [np.array(a, dtype=np.int64) for a in (comp, dst, src, val)]


def _ring_ops(z):
    kinds = z["ring_kind"]
    return [np.zeros(len(kinds), dtype=np.int64), z["ring_dst"].astype(np.int64),
            np.where(kinds == 2, z["ring_src"], -1).astype(np.int64),
            np.where(kinds == 1, np.arange(len(kinds)), -1).astype(np.int64)]


def _outflow_flux(z, F):
    """ApplyOutflowFlux in the reference's summation order, as k_bc_outflow does it."""
    nin, nout = len(z["inlet_comp"]), len(z["outflow_comp"])
    if not nout:
        return
    q_in = 0.0
    for q in range(nin):
        q_in -= z["inlet_sign"][q] * F[z["inlet_comp"][q]][z["inlet_index"][q]] * z["inlet_area"][q]
    q_out = a_out = 0.0
    for q in range(nout):
        q_out += z["outflow_sign"][q] * F[z["outflow_comp"][q]][z["outflow_index"][q]] * z["outflow_area"][q]
        a_out += z["outflow_area"][q]
    if a_out <= 0.0:
        return
    delta = (q_in - q_out) / a_out
    for q in range(nout):
        g = F[z["outflow_comp"][q]]
        x = g[z["outflow_index"][q]] + z["outflow_sign"][q] * delta
        g[z["outflow_index"][q]] = x
        g[z["outflow_outer"][q]] = x


@pytest.mark.parametrize("name", NAMES)
def test_planned_levels_without_boundary_functions_match_oracle(lib, name):
    """The same levels with the prescribed writes left out (no velocity function) and 0 at the prescribed ring
    entries (no pressure function): the oracle's serial replay under the same conditions."""
    from nereus_cfd_b200.boundary import plan_levels

    case, meta, z = load_golden(name)
    vel, pres, _, _ = plan_levels(dict(z), *_dims(case))
    u, v, p = z["u_in"].copy(), z["v_in"].copy(), z["p_in"].copy()
    w = z["w_in"].copy() if len(z["w_in"]) else np.zeros(1)
    _run_levels(_velocity_ops(z), vel, [u, v, w], None, False)
    _outflow_flux(z, [u, v, w])
    _run_levels(_ring_ops(z), pres, [p], None, True)
    lists = dict(z)
    lists["ring_value"] = np.zeros_like(z["ring_value"])
    ru, rv, rw, rp = cpu.bc_replay(lists, z["u_in"], z["v_in"], z["w_in"], z["p_in"], with_velocity_function=False)
    assert np.array_equal(p, rp)
    assert np.array_equal(u, ru) and np.array_equal(v, rv)
    if len(z["w_in"]):
        assert np.array_equal(w, rw)


@pytest.mark.parametrize("name", NAMES)
def test_planned_levels_reproduce_the_reference(lib, name):
    """The levels the library plans (nereus_b200_bc_plan, the code nereus_b200_bc_create runs), executed level by
    level as parallel scatters, leave the reference's fields bit for bit."""
    from nereus_cfd_b200.boundary import plan_levels

    case, meta, z = load_golden(name)
    vel, pres, nv, npl = plan_levels(dict(z), *_dims(case))
    assert nv == (int(vel.max()) + 1 if len(vel) else 0) and npl == (int(pres.max()) + 1 if len(pres) else 0)
    u, v, p = z["u_in"].copy(), z["v_in"].copy(), z["p_in"].copy()
    w = z["w_in"].copy() if len(z["w_in"]) else np.zeros(1)
    ops = _velocity_ops(z)
    assert len(vel) == len(ops[0])
    _run_levels(ops, vel, [u, v, w], z["presc_value"], False)
    _outflow_flux(z, [u, v, w])
    _run_levels(_ring_ops(z), pres, [p], z["ring_value"], True)
    assert np.array_equal(u, z["u_out"]) and np.array_equal(v, z["v_out"]) and np.array_equal(p, z["p_out"])
    if len(z["w_in"]):
        assert np.array_equal(w, z["w_out"])
