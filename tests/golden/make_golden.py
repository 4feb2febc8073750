"""Writes the golden fixtures under tests/golden/ from the NEREUS reference's own pressure path.

Run in a checkout that has the reference sources (it builds oracle/_ref/ref_harness from them first):

    python tests/golden/make_golden.py [REF_ROOT] [--only explicit|flip|bc|<fixture name>]

Each fixture is one small case: the inputs both sides read (face velocities, the prescribed ring pressure) and what
the reference computed from them (cell types, IDP, the CSR matrix, b before and after the compatibility step, the
Eigen-CG solution, the pressure field, the projected velocities, iterations, relative residual, max |div u|, and its
spacing tables). The case geometry itself is rebuilt from the builder name and arguments stored in ``meta``.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from nereus_cfd_b200 import workloads as W  # noqa: E402
from oracle import refcase  # noqa: E402

# (fixture name, builder, kwargs, solver tolerance or None for the case's own)
CASES = [
    ("closed_box_2d_16", "closed_box_2d", {"n": 16, "seed": 11}, 1e-12),
    ("sphere_outlet_3d_12", "sphere_outlet_3d", {"n": 12, "seed": 12}, 1e-12),
    ("stretched_cylinder_3d_24x16x16", "stretched_cylinder_3d", {"nx": 24, "ny": 16, "nz": 16, "seed": 13}, 1e-12),
    ("flip_tank_3d_12", "flip_tank_3d", {"n": 12, "seed": 14}, 1e-12),
    ("dirichlet_linear_2d_40", "dirichlet_linear_2d", {"n": 40}, None),
    ("dirichlet_linear_3d_20", "dirichlet_linear_3d", {"n": 20}, None),
    ("channel_2d_stretched_24x12", "channel_2d_stretched", {"nx": 24, "ny": 12, "seed": 15}, 1e-12),
    ("inflow_outflow_3d_8", "inflow_outflow_3d", {"n": 8, "seed": 16}, 1e-12),
    ("all_solid_3d_6", "all_solid_3d", {"n": 6, "seed": 17}, 1e-12),
    # the 2D 128^2 closed box at full size (all-Neumann, compatibility on; the case's own tolerance is 1e-10)
    ("closed_box_2d_128", "closed_box_2d", {"n": 128, "seed": 1}, 1e-12),
]


# the schemes with a previous step: (fixture name, builder, kwargs, tol, scheme, time of the new step)
SCHEME_CASES = [
    ("incremental_pressure_outlet_3d_12", "pressure_outlet_3d", {"n": 12, "seed": 18}, 1e-12,
     refcase.SCHEME_INCREMENTAL, 0.3),
    ("incremental_closed_box_2d_16", "closed_box_2d", {"n": 16, "seed": 19}, 1e-12, refcase.SCHEME_INCREMENTAL, 0.0),
    ("warm_sphere_outlet_3d_12", "sphere_outlet_3d", {"n": 12, "seed": 20}, 1e-12, refcase.SCHEME_CHORIN_WARM, 0.0),
]


# the EXPLICIT method's own pressure step and projection (2D, uniform): (fixture name, builder, kwargs, SOR tolerance
# relative to max |b| in the max norm)
EXPLICIT_CASES = [
    ("explicit_cavity_outlet_2d_32", "cavity_outlet_2d", {"n": 32, "seed": 21}, 1e-13),
    ("explicit_closed_box_2d_16", "closed_box_2d", {"n": 16, "seed": 22}, 1e-13),
]
# a scene outside the equivalence: air (EMPTY) cells inside the grid, toward which EXPLICIT's coefficient is 2 and the
# shared system's ring factor 1
EXPLICIT_LIMIT_CASES = [
    ("limit_explicit_tank_2d_24", "flip_tank_2d", {"n": 24, "seed": 28}, 1e-13),
]


# FLIP's re-labelling from particles, then the Chorin step on the new labels: (fixture name, builder, kwargs,
# particle seed, particles per cell)
FLIP_CASES = [
    ("flip_relabel_tank_3d_16", "flip_tank_3d", {"n": 16, "seed": 41}, 57, 4),
    ("flip_relabel_tank_2d_24", "flip_tank_2d", {"n": 24, "seed": 32}, 56, 4),
]


# the boundary-condition replay (EnforceVelocityBC + EnforcePressureBC) on seeded N(0,1) fields: (fixture name,
# builder, kwargs, time)
BC_CASES = [
    ("bc_channel_3d_12", "bc_channel_3d", {"n": 12, "seed": 23}, 0.3),
    ("bc_outlet_2d_20", "bc_outlet_2d", {"n": 20, "seed": 24}, 0.7),
    ("bc_inflow_outflow_3d_8", "inflow_outflow_3d", {"n": 8, "seed": 25}, 0.1),
    ("bc_pressure_outlet_3d_12", "pressure_outlet_3d", {"n": 12, "seed": 26}, 0.45),
    ("bc_sphere_outlet_3d_10", "sphere_outlet_3d", {"n": 10, "seed": 27}, 0.0),
] + [("bc_suite_scene%d_%dd" % (k, d), "bc_suite_scene", {"scene": k, "dim": d, "seed": 30 + 2 * k + d}, t)
     for k in range(4) for d, t in ((3, 0.25), (2, 0.6))] + [  # the reference's own boundary test scenes
    ("bc_suite_scene%d_%dd_stretched" % (k, d), "bc_suite_scene",
     {"scene": k, "dim": d, "seed": 40 + 2 * k + d, "stretched": True}, 0.45) for k in (1, 3) for d in (3, 2)]


def build_case(builder: str, kwargs: dict) -> W.Case:
    return getattr(W, builder)(**kwargs)


def previous_step(case, types, u, v, w, scheme, time):
    """p^n for a scheme case: seeded interior values with the outlet's p_b at t - dt (incremental), or the cold
    Chorin solution plus a 1e-3 N(0,1) perturbation on the unknowns (warm start: a guess close to the answer)."""
    g = case.grid
    if scheme == refcase.SCHEME_INCREMENTAL:
        ring = W.outlet_pressure(time - case.dt) if case.scene.pressure_expr == W.PRESSURE_OUTLET_EXPR else None
        return W.previous_pressure(g, types, case.seed, ring)
    cold = refcase.run(case, u, v, w, tol=1e-12)
    noise = W.previous_pressure(g, types, case.seed)
    return cold.p + 1e-3 * noise


def write_scheme_case(name, builder, kwargs, tol, scheme, time):
    case = build_case(builder, kwargs)
    g = case.grid
    probe = refcase.run(case, *[np.zeros(int(np.prod(s))) if s != (0,) else np.zeros(0)
                                for s in (g.u_shape(), g.v_shape(), g.w_shape())], tol=1e-6)
    types = probe.types
    u, v, w = W.face_velocities(g, types, case.seed, case.velocity_rule, case.fp32_velocity)
    p_prev = previous_step(case, types, u, v, w, scheme, time)
    ref = refcase.run(case, u, v, w, tol=tol, scheme=scheme, p_prev=p_prev, time=time)
    cold = refcase.run(case, u, v, w, tol=tol, time=time)
    p_in = np.where(ref.types == W.PRESSURE, ref.p_final, 0.0)
    meta = dict(name=name, builder=builder, kwargs=kwargs, tol=tol, needs_compat=case.needs_compat, rho=case.rho,
                dt=case.dt, n=ref.n, iters=ref.iters, cold_iters=cold.iters, singular=ref.singular,
                rel_res=ref.rel_res, max_div=ref.max_div, dh=ref.dh, scheme=scheme, time=time,
                ref_norm=ref.ref_norm)
    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(
        out, meta=np.array(json.dumps(meta)), u=u.ravel(), v=v.ravel(), w=w.ravel(), p_in=p_in, p_prev=p_prev,
        types=ref.types, idp=ref.idp, b_raw=ref.b_raw, b=ref.b, x=ref.x, p=ref.p, p_final=ref.p_final,
        u_out=ref.u, v_out=ref.v, w_out=ref.w)
    print("%-36s n=%-6d iters=%-4d (cold %d) rel_res=%.2e max_div=%.2e ref_norm=%.3g  %d KB" % (
        name, ref.n, ref.iters, cold.iters, ref.rel_res, ref.max_div, ref.ref_norm, os.path.getsize(out) // 1024))


def write_explicit_case(name, builder, kwargs, tol):
    """The reference's Explicit2D::Pressure + Projection on a uniform 2D case, with the shared assembly's IDP, b and
    matrix beside it (rel_res: the SOR solution's relative residual in that system)."""
    case = build_case(builder, kwargs)
    g = case.grid
    probe = refcase.run(case, np.zeros(int(np.prod(g.u_shape()))), np.zeros(int(np.prod(g.v_shape()))), np.zeros(0),
                        tol=1e-6)
    types = probe.types
    u, v, w = W.face_velocities(g, types, case.seed, case.velocity_rule, case.fp32_velocity)
    ref = refcase.run(case, u, v, w, tol=tol, max_iters=2000000, scheme=refcase.SCHEME_EXPLICIT)
    p_in = np.where(ref.types == W.PRESSURE, ref.p, 0.0)
    meta = dict(name=name, builder=builder, kwargs=kwargs, tol=tol, needs_compat=case.needs_compat, rho=case.rho,
                dt=case.dt, n=ref.n, singular=ref.singular, rel_res=ref.rel_res, max_div=ref.max_div, dh=ref.dh,
                scheme=refcase.SCHEME_EXPLICIT)
    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(
        out, meta=np.array(json.dumps(meta)), u=u.ravel(), v=v.ravel(), w=w.ravel(), p_in=p_in, types=ref.types,
        idp=ref.idp, b=ref.b, x=ref.x, p=ref.p, u_out=ref.u, v_out=ref.v)
    print("%-36s n=%-6d rel_res=%.2e max_div=%.2e singular=%d  %d KB" % (
        name, ref.n, ref.rel_res, ref.max_div, ref.singular, os.path.getsize(out) // 1024))


def write_flip_case(name, builder, kwargs, particle_seed, ppc):
    """The reference's FLIP{2,3}D::UpdateFluidCells from seeded particles (W.flip_particles) on the scene's labels,
    then its Chorin step on the new labels."""
    case = build_case(builder, kwargs)
    g = case.grid
    probe = refcase.run(case, *[np.zeros(int(np.prod(s))) if s != (0,) else np.zeros(0)
                                for s in (g.u_shape(), g.v_shape(), g.w_shape())], tol=1e-6)
    xyz = W.flip_particles(case, probe.types, particle_seed, ppc)
    u, v, w = W.face_velocities(g, probe.types, case.seed, case.velocity_rule, case.fp32_velocity)
    tol = 1e-12
    ref = refcase.run(case, u, v, w, tol=tol, scheme=refcase.SCHEME_FLIP_RELABEL, particles=xyz)
    assert np.array_equal(ref.types_before, probe.types)
    p_in = np.where(ref.types == W.PRESSURE, ref.p, 0.0)
    meta = dict(name=name, builder=builder, kwargs=kwargs, particle_seed=particle_seed, ppc=ppc, tol=tol,
                needs_compat=case.needs_compat, rho=case.rho, dt=case.dt, n=ref.n, iters=ref.iters,
                singular=ref.singular, rel_res=ref.rel_res, max_div=ref.max_div, dh=ref.dh,
                origin=[float(o) for o in ref.origin], scheme=refcase.SCHEME_FLIP_RELABEL)
    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(
        out, meta=np.array(json.dumps(meta)), xyz=xyz, types_in=ref.types_before, u=u.ravel(), v=v.ravel(),
        w=w.ravel(), p_in=p_in, types=ref.types, idp=ref.idp, b=ref.b, x=ref.x, p=ref.p, u_out=ref.u, v_out=ref.v,
        w_out=ref.w)
    changed = int((ref.types != ref.types_before).sum())
    print("%-36s particles=%-6d relabelled=%-5d n=%-6d rel_res=%.2e  %d KB" % (
        name, xyz.shape[0], changed, ref.n, ref.rel_res, os.path.getsize(out) // 1024))


def write_bc_case(name, builder, kwargs, time):
    """The reference's EnforceVelocityBC and EnforcePressureBC on seeded fields: its lists (with the values its
    boundary functions gave at `time`) and the fields before and after."""
    case = build_case(builder, kwargs)
    g = case.grid
    seed = kwargs["seed"]
    u = W.normals(W.stream_seed(seed, 10), int(np.prod(g.u_shape())))
    v = W.normals(W.stream_seed(seed, 11), int(np.prod(g.v_shape())))
    w = W.normals(W.stream_seed(seed, 12), int(np.prod(g.w_shape()))) if g.dim == 3 else np.zeros(0)
    p = W.normals(W.stream_seed(seed, 13), g.cells)
    r = refcase.run_bc(case, u, v, w, p, time)
    meta = dict(name=name, builder=builder, kwargs=kwargs, time=time)
    arrays = {k: val for k, val in r.items() if isinstance(val, np.ndarray) and k not in ("u", "v", "w", "p")}
    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(out, meta=np.array(json.dumps(meta)), u_in=u, v_in=v, w_in=w, p_in=p, u_out=r["u"],
                        v_out=r["v"], w_out=r["w"], p_out=r["p"], **arrays)
    print("%-36s presc=%-5d copies=%-5d ring=%-5d outflow=%-4d  %d KB" % (
        name, len(r["presc_comp"]), len(r["copy_comp"]), len(r["ring_dst"]), len(r["outflow_comp"]),
        os.path.getsize(out) // 1024))


def main(ref_root: str = "/root/reference", only: str = "") -> None:
    if not refcase.build(ref_root):
        raise SystemExit("the reference harness could not be built from %s" % ref_root)
    if only == "explicit":
        for args in EXPLICIT_CASES + EXPLICIT_LIMIT_CASES:
            write_explicit_case(*args)
        return
    if only == "flip":
        for args in FLIP_CASES:
            write_flip_case(*args)
        return
    if only == "bc":
        for args in BC_CASES:
            write_bc_case(*args)
        return
    for name, builder, kwargs, tol in CASES:
        if only and only != name:
            continue
        case = build_case(builder, kwargs)
        g = case.grid
        # labels from the reference's own scene code (label_mode 0), then velocities from those labels
        probe = refcase.run(case, *[np.zeros(int(np.prod(s))) if s != (0,) else np.zeros(0)
                                    for s in (g.u_shape(), g.v_shape(), g.w_shape())], tol=1e-6)
        types = probe.types
        u, v, w = W.face_velocities(g, types, case.seed, case.velocity_rule, case.fp32_velocity)
        ref = refcase.run(case, u, v, w, tol=tol if tol is not None else case.tol)
        p_in = np.where(ref.types == W.PRESSURE, ref.p, 0.0)
        meta = dict(name=name, builder=builder, kwargs=kwargs, tol=tol if tol is not None else case.tol,
                    needs_compat=case.needs_compat, rho=case.rho, dt=case.dt, n=ref.n, iters=ref.iters,
                    singular=ref.singular, rel_res=ref.rel_res, max_div=ref.max_div, dh=ref.dh)
        out = os.path.join(HERE, name + ".npz")
        np.savez_compressed(
            out, meta=np.array(json.dumps(meta)), u=u.ravel(), v=v.ravel(), w=w.ravel(), p_in=p_in,
            types=ref.types, idp=ref.idp, rowptr=ref.rowptr, col=ref.col, val=ref.val, b_raw=ref.b_raw, b=ref.b,
            x=ref.x, p=ref.p, u_out=ref.u, v_out=ref.v, w_out=ref.w,
            **{"width%d" % a: ref.width[a] for a in range(3)}, **{"gap%d" % a: ref.gap[a] for a in range(3)},
            **{"centre%d" % a: ref.centre[a] for a in range(3)})
        print("%-36s n=%-6d iters=%-4d rel_res=%.2e max_div=%.2e  %d KB" % (
            name, ref.n, ref.iters, ref.rel_res, ref.max_div, os.path.getsize(out) // 1024))
    if only:
        return
    for args in SCHEME_CASES:
        write_scheme_case(*args)
    for args in EXPLICIT_CASES + EXPLICIT_LIMIT_CASES:
        write_explicit_case(*args)
    for args in FLIP_CASES:
        write_flip_case(*args)
    for args in BC_CASES:
        write_bc_case(*args)


if __name__ == "__main__":
    argv = sys.argv[1:]
    only = ""
    if "--only" in argv:
        k = argv.index("--only")
        only = argv[k + 1]
        argv = argv[:k] + argv[k + 2:]
    main(*argv, only=only)
