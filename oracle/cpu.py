"""ORACLE / TEST INFRASTRUCTURE ONLY: ctypes wrapper of the plain-C restatement ``oracle/pressure_oracle.c``.

``solve_projection`` runs the reference's pressure step end to end the way PressureSolver3D::SolveScheme and
ProjectPressure do (src/Methods/PPESolver/PressureSolver3D.cpp:279-328, 417-438): assemble, right-hand side,
compatibility, Eigen-style diagonal-PCG, level, scatter, ring, projection.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_u8 = ctypes.POINTER(ctypes.c_uint8)


class OrGrid(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int),
                ("nonuniform", ctypes.c_int), ("dh", ctypes.c_double),
                ("width", _dp * 3), ("gap", _dp * 3), ("types", _u8)]


class OrRegion(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("region", ctypes.c_int), ("axis", ctypes.c_int), ("invert", ctypes.c_int),
                ("p0", ctypes.c_double * 3), ("p1", ctypes.c_double * 3), ("radius", ctypes.c_double)]


class OrScene(ctypes.Structure):
    _fields_ = [("face_kind", ctypes.c_int * 6), ("face_has_p", ctypes.c_int * 6), ("face_order", ctypes.c_int * 6),
                ("nregions", ctypes.c_int), ("regions", OrRegion * 16)]


def build() -> str:
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "pressure_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    return path


def lib():
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(build())
        L = _LIB
        L.or_label_cells.argtypes = [ctypes.c_int] * 4 + [_dp, _dp, _dp, ctypes.POINTER(OrScene), _u8]
        L.or_number_unknowns.argtypes = [ctypes.POINTER(OrGrid), _ip]
        L.or_number_unknowns.restype = ctypes.c_int
        L.or_assemble.argtypes = [ctypes.POINTER(OrGrid), _ip, _ip, _ip, _dp, ctypes.POINTER(ctypes.c_int)]
        L.or_assemble.restype = ctypes.c_int
        L.or_rhs.argtypes = [ctypes.POINTER(OrGrid), _ip, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, _dp]
        L.or_compat.argtypes = [_dp, ctypes.c_int]
        L.or_cg.argtypes = [_ip, _ip, _dp, ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_int, _dp]
        L.or_cg.restype = ctypes.c_int
        L.or_level_mean.argtypes = [_dp, ctypes.c_int]
        L.or_scatter.argtypes = [ctypes.POINTER(OrGrid), _ip, _dp, _dp]
        L.or_ring_replay.argtypes = [ctypes.POINTER(OrGrid), _dp]
        L.or_project.argtypes = [ctypes.POINTER(OrGrid), _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double]
        L.or_max_divergence.argtypes = [ctypes.POINTER(OrGrid), _dp, _dp, _dp]
        L.or_max_divergence.restype = ctypes.c_double
        L.or_residual_norm.argtypes = [_ip, _ip, _dp, ctypes.c_int, _dp, _dp]
        L.or_residual_norm.restype = ctypes.c_double
        L.or_update_fluid_cells.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 4 + [_dp, ctypes.c_longlong, _u8]
        L.or_update_fluid_cells.restype = ctypes.c_longlong
        _i = ctypes.POINTER(ctypes.c_int32)
        L.or_bc_velocity.argtypes = ([_dp] * 3 + [_i] * 4 + [_i, _i, _dp, ctypes.c_int] + [_i] * 3 + [ctypes.c_int] +
                                     [_i, _i, _dp, _dp, ctypes.c_int] + [_i] * 3 + [_dp, _dp, ctypes.c_int])
        L.or_bc_pressure.argtypes = [_dp, _i, _i, _i, _dp, ctypes.c_int]
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(t)


class GridView:
    """Keeps the arrays an OrGrid points at alive."""

    def __init__(self, grid, types: np.ndarray):
        self.widths = [np.ascontiguousarray(w, dtype=np.float64) for w in grid.width_tables()]
        self.gaps = [np.ascontiguousarray(g, dtype=np.float64) for g in grid.gap_tables()]
        self.types = np.ascontiguousarray(types.reshape(-1), dtype=np.uint8)
        self.s = OrGrid()
        self.s.dim, self.s.Nx, self.s.Ny, self.s.Nz = grid.dim, grid.Nx, grid.Ny, grid.Nz
        self.s.nonuniform = int(grid.nonuniform)
        self.s.dh = grid.dh
        for a in range(3):
            self.s.width[a] = _p(self.widths[a], _dp)
            self.s.gap[a] = _p(self.gaps[a], _dp)
        self.s.types = _p(self.types, _u8)
        self.grid = grid

    @property
    def ref(self):
        return ctypes.byref(self.s)


def scene_struct(scene) -> OrScene:
    s = OrScene()
    kind, has_p, order = scene.face_arrays()
    for f in range(6):
        s.face_kind[f], s.face_has_p[f], s.face_order[f] = kind[f], has_p[f], order[f]
    s.nregions = len(scene.regions)
    for n, r in enumerate(scene.regions):
        s.regions[n].kind, s.regions[n].region, s.regions[n].axis = r.kind, r.region, r.axis
        s.regions[n].invert = int(r.invert)
        for a in range(3):
            s.regions[n].p0[a], s.regions[n].p1[a] = r.p0[a], r.p1[a]
        s.regions[n].radius = r.radius
    return s


def label_cells(grid, scene) -> np.ndarray:
    cx, cy, cz = [np.ascontiguousarray(c, dtype=np.float64) for c in grid.sample_coords(scene.at_centre)]
    out = np.zeros(grid.cells, dtype=np.uint8)
    s = scene_struct(scene)
    lib().or_label_cells(grid.dim, grid.Nx, grid.Ny, grid.Nz if grid.dim == 3 else 1, _p(cx, _dp), _p(cy, _dp),
                         _p(cz, _dp), ctypes.byref(s), _p(out, _u8))
    return out


def update_fluid_cells(grid, types, xyz, origin, dh=None):
    """FLIP's re-labelling from particle positions (``or_update_fluid_cells``): returns the new cell types and the
    number of particles skipped as out of range. xyz: (count, 3) float64 positions; origin: FacePos(X|Y|Z, 0)."""
    out = np.ascontiguousarray(types, dtype=np.uint8).reshape(-1).copy()
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    dh = grid.dh if dh is None else dh
    oz = origin[2] if len(origin) > 2 else 0.0
    skipped = lib().or_update_fluid_cells(grid.dim, grid.Nx, grid.Ny, grid.Nz if grid.dim == 3 else 1,
                                          origin[0], origin[1], oz, dh, _p(xyz, _dp), xyz.shape[0], _p(out, _u8))
    return out, int(skipped)


def bc_replay(lists, u, v, w, p, with_velocity_function=True):
    """EnforceVelocityBC + EnforcePressureBC from the reference's lists (``lists``: the arrays of a bc_* fixture, or
    what refcase.run_bc returned): new copies of u, v, w, p."""
    L = lib()
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    _i = ctypes.POINTER(ctypes.c_int32)
    u, v, p = f64(u).copy(), f64(v).copy(), f64(p).copy()
    two_d = len(w) == 0
    w = np.zeros(1) if two_d else f64(w).copy()
    keep = []

    def P(a, t):
        keep.append(a)
        return a.ctypes.data_as(t)
    solid = [i32(lists["solid%d" % c]) for c in range(3)]
    nsolid = np.array([len(x) for x in solid], dtype=np.int32)
    pv = f64(lists["presc_value"]) if with_velocity_function else None
    L.or_bc_velocity(P(u, _dp), P(v, _dp), P(w, _dp), P(solid[0], _i), P(solid[1], _i), P(solid[2], _i),
                     P(nsolid, _i), P(i32(lists["presc_comp"]), _i), P(i32(lists["presc_index"]), _i),
                     P(pv, _dp) if pv is not None else None, len(lists["presc_comp"]),
                     P(i32(lists["copy_comp"]), _i), P(i32(lists["copy_dst"]), _i), P(i32(lists["copy_src"]), _i),
                     len(lists["copy_comp"]), P(i32(lists["inlet_comp"]), _i), P(i32(lists["inlet_index"]), _i),
                     P(f64(lists["inlet_area"]), _dp), P(f64(lists["inlet_sign"]), _dp), len(lists["inlet_comp"]),
                     P(i32(lists["outflow_comp"]), _i), P(i32(lists["outflow_index"]), _i),
                     P(i32(lists["outflow_outer"]), _i), P(f64(lists["outflow_area"]), _dp),
                     P(f64(lists["outflow_sign"]), _dp), len(lists["outflow_comp"]))
    L.or_bc_pressure(P(p, _dp), P(i32(lists["ring_dst"]), _i), P(i32(lists["ring_kind"]), _i),
                     P(i32(lists["ring_src"]), _i), P(f64(lists["ring_value"]), _dp), len(lists["ring_dst"]))
    return u, v, (np.zeros(0) if two_d else w), p


@dataclass
class Assembly:
    idp: np.ndarray
    n: int
    rowptr: np.ndarray
    col: np.ndarray
    val: np.ndarray
    singular: bool


def assemble(gv: GridView) -> Assembly:
    L = lib()
    idp = np.zeros(gv.grid.cells, dtype=np.int32)
    n = L.or_number_unknowns(gv.ref, _p(idp, _ip))
    cap = 7 * max(n, 1)
    rowptr = np.zeros(n + 1, dtype=np.int32)
    col = np.zeros(cap, dtype=np.int32)
    val = np.zeros(cap, dtype=np.float64)
    sing = ctypes.c_int(0)
    nnz = L.or_assemble(gv.ref, _p(idp, _ip), _p(rowptr, _ip), _p(col, _ip), _p(val, _dp), ctypes.byref(sing))
    return Assembly(idp, n, rowptr, col[:nnz].copy(), val[:nnz].copy(), bool(sing.value))


def rhs(gv: GridView, asm: Assembly, u, v, w, p, rho, dt) -> np.ndarray:
    b = np.zeros(max(asm.n, 1))
    w = w if w.size else np.zeros(1)
    lib().or_rhs(gv.ref, _p(asm.idp, _ip), _p(u, _dp), _p(v, _dp), _p(w, _dp), _p(p, _dp), rho, dt, _p(b, _dp))
    return b[: asm.n]


def compat(b: np.ndarray) -> np.ndarray:
    b = np.ascontiguousarray(b, dtype=np.float64).copy()
    if b.size:
        lib().or_compat(_p(b, _dp), b.size)
    return b


def cg(asm: Assembly, b: np.ndarray, tol: float, max_iters: int = 1000000):
    x = np.zeros(max(asm.n, 1))
    bb = np.ascontiguousarray(b, dtype=np.float64)
    if asm.n == 0:
        return x[:0], 0, 0.0
    err = ctypes.c_double(0.0)
    it = lib().or_cg(_p(asm.rowptr, _ip), _p(asm.col, _ip), _p(asm.val, _dp), asm.n, _p(bb, _dp), _p(x, _dp), tol,
                     max_iters, ctypes.byref(err))
    return x, it, err.value


def residual_norm(asm: Assembly, b, x) -> float:
    return lib().or_residual_norm(_p(asm.rowptr, _ip), _p(asm.col, _ip), _p(asm.val, _dp), asm.n,
                                  _p(np.ascontiguousarray(b), _dp), _p(np.ascontiguousarray(x), _dp))


@dataclass
class Projection:
    types: np.ndarray
    asm: Assembly
    b_raw: np.ndarray
    b: np.ndarray
    x: np.ndarray
    iters: int
    rel_res: float
    p: np.ndarray
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    max_div: float


def solve_projection(grid, types, u, v, w, p_in, rho, dt, needs_compat, tol, max_iters=1000000) -> Projection:
    """The reference's Chorin pressure step + projection, restated (see the module docstring)."""
    gv = GridView(grid, types)
    asm = assemble(gv)
    p = np.ascontiguousarray(p_in, dtype=np.float64).copy()
    lib().or_ring_replay(gv.ref, _p(p, _dp))  # EnforcePressureBC before the solve
    b_raw = rhs(gv, asm, u, v, w, p, rho, dt)
    b = compat(b_raw) if (needs_compat and asm.singular and asm.n > 0) else b_raw.copy()
    x, it, err = cg(asm, b, tol, max_iters)
    x = x[: asm.n].copy()
    if needs_compat and asm.singular and asm.n > 0:
        lib().or_level_mean(_p(x, _dp), asm.n)
    xs = x if x.size else np.zeros(1)
    lib().or_scatter(gv.ref, _p(asm.idp, _ip), _p(xs, _dp), _p(p, _dp))
    lib().or_ring_replay(gv.ref, _p(p, _dp))
    uu, vv = u.copy(), v.copy()
    ww = w.copy() if w.size else np.zeros(1)
    lib().or_project(gv.ref, _p(uu, _dp), _p(vv, _dp), _p(ww, _dp), _p(p, _dp), rho, dt)
    md = lib().or_max_divergence(gv.ref, _p(uu, _dp), _p(vv, _dp), _p(ww, _dp))
    bn = float(np.linalg.norm(b))
    rr = residual_norm(asm, b, x) / bn if bn > 0 else 0.0
    return Projection(gv.types.copy(), asm, b_raw, b, x, it, rr, p, uu, vv, ww if w.size else w, md)


PRESSURE = 4


def solve_scheme(grid, types, u, v, w, p_in, p_prev, rho, dt, needs_compat, tol, incremental, warm=False,
                 max_iters=1000000) -> Projection:
    """The step with a previous pressure p_prev, restated from the reference:
    incremental (SolveScheme with `old`, PressureSolver3D.cpp:262-328, then Project :396-401 =
    ProjectPressure + AccumulatePressureIncrement :374-393): DirichletSum reads p_b(t^{n+1}) - p_b(t^n) on PRESSURE
    cells; the Eigen CG stops at ||r|| < tol max(||b||, ||b + A p^n||) (SolveEigenPressure, PressureSettings.h:
    411-427); phi is not levelled; the ring carries phi; the velocity takes grad phi; p = p^n + phi on the unknowns,
    levelled, and EnforcePressureBC puts the prescribed ring back.
    warm (Chorin, BuildWarmStartGuess :222-244): the CG starts from p_prev on the unknowns, mean-free when the
    compatibility condition applies. Returns the Projection with p = the final pressure; .x is the solve's result."""
    gv = GridView(grid, types)
    asm = assemble(gv)
    sing = needs_compat and asm.singular and asm.n > 0
    p = np.ascontiguousarray(p_in, dtype=np.float64).copy()
    lib().or_ring_replay(gv.ref, _p(p, _dp))
    ring_entry = p.copy()
    prev = np.ascontiguousarray(p_prev, dtype=np.float64)
    t = gv.types
    known = np.where(t == PRESSURE, p - prev, 0.0) if incremental else p
    b_raw = rhs(gv, asm, u, v, w, np.ascontiguousarray(known), rho, dt)
    b = compat(b_raw) if sing else b_raw.copy()
    idp = asm.idp
    on = idp >= 0
    pn = np.zeros(max(asm.n, 1))
    pn[idp[on]] = prev[on]
    pn = pn[: asm.n]
    x = np.zeros(max(asm.n, 1))
    it, tol_eff, solve = 0, tol, asm.n > 0
    if incremental and asm.n > 0:
        ref = float(np.linalg.norm(b + spmv(asm, pn)))
        bn = float(np.linalg.norm(b))
        if ref > 0.0:
            if bn <= tol * ref:
                solve = False
            else:
                tol_eff = min(0.5, tol * ref / bn)
    if warm and asm.n > 0 and not grid.nonuniform:
        x[: asm.n] = pn
        if sing:
            x[: asm.n] -= x[: asm.n].mean()
    if solve:
        err = ctypes.c_double(0.0)
        it = lib().or_cg(_p(asm.rowptr, _ip), _p(asm.col, _ip), _p(asm.val, _dp), asm.n,
                         _p(np.ascontiguousarray(b), _dp), _p(x, _dp), tol_eff, max_iters, ctypes.byref(err))
    x = x[: asm.n].copy()
    if sing and not incremental:
        lib().or_level_mean(_p(x, _dp), asm.n)
    xs = x if x.size else np.zeros(1)
    lib().or_scatter(gv.ref, _p(idp, _ip), _p(xs, _dp), _p(p, _dp))
    lib().or_ring_replay(gv.ref, _p(p, _dp))
    if incremental:
        p = np.where(t == PRESSURE, p - prev, p)
    uu, vv = u.copy(), v.copy()
    ww = w.copy() if w.size else np.zeros(1)
    lib().or_project(gv.ref, _p(uu, _dp), _p(vv, _dp), _p(ww, _dp), _p(p, _dp), rho, dt)
    md = lib().or_max_divergence(gv.ref, _p(uu, _dp), _p(vv, _dp), _p(ww, _dp))
    if incremental:
        acc = np.zeros(max(asm.n, 1))
        acc[idp[on]] = prev[on] + p[on]
        acc = acc[: asm.n].copy()
        if sing:
            lib().or_level_mean(_p(acc, _dp), asm.n)
        accs = acc if acc.size else np.zeros(1)
        lib().or_scatter(gv.ref, _p(idp, _ip), _p(accs, _dp), _p(p, _dp))
        p = np.where(t == PRESSURE, ring_entry, p)
        lib().or_ring_replay(gv.ref, _p(p, _dp))
    bn = float(np.linalg.norm(b))
    rr = residual_norm(asm, b, x) / bn if bn > 0 else 0.0
    return Projection(t.copy(), asm, b_raw, b, x, it, rr, p, uu, vv, ww if w.size else w, md)


def spmv(asm: Assembly, x: np.ndarray) -> np.ndarray:
    """A x with the assembled CSR (rows in order, each row's entries in column order)."""
    y = np.zeros(asm.n)
    for r in range(asm.n):
        a, b = asm.rowptr[r], asm.rowptr[r + 1]
        y[r] = np.dot(asm.val[a:b], x[asm.col[a:b]])
    return y


def ring_replay(grid, types, p):
    gv = GridView(grid, types)
    p = np.ascontiguousarray(p, dtype=np.float64).copy()
    lib().or_ring_replay(gv.ref, _p(p, _dp))
    return p


def max_divergence(grid, types, u, v, w) -> float:
    gv = GridView(grid, types)
    ww = w if w.size else np.zeros(1)
    return lib().or_max_divergence(gv.ref, _p(np.ascontiguousarray(u), _dp), _p(np.ascontiguousarray(v), _dp),
                                   _p(np.ascontiguousarray(ww), _dp))
