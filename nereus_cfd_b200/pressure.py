"""The reference's pressure-solver interface over the B200 library.

``PressureSolver`` mirrors the static API of NEREUS's PressureSolver2D / PressureSolver3D
(src/Methods/PPESolver/PressureSolver3D.h:49-75): InitializePressureSolver, Destroy/ReleasePressureSolver,
SolvePressure, SolveLaplacian, SystemSize, LastIterations, ProjectPressure, GetIDP -- same names, same argument
meaning, same error behaviour (SolveLaplacian returns False on a size mismatch; a solve that does not converge
reports it and keeps the last iterate). It calls the C ABI of include/nereus_b200.h; nothing here computes.

The B200 pressure step is fused: SolvePressure runs the right-hand side, solve, level, scatter, ring AND the
velocity correction on the device in one call (nothing runs between the reference's "pressure" step at order 4
and its "projection" step at order 6), so ProjectPressure only confirms that it has been done.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional

import numpy as np

from . import capi
from .workloads import Grid


@dataclasses.dataclass
class MACGrid:
    """A MAC grid's state as the pressure step sees it: geometry, cell types and the face/centre fields in the
    reference's layouts (float64, flat). ``p`` carries the prescribed ring values (MAC::EnforcePressureBC)."""

    grid: Grid
    types: np.ndarray
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    p: np.ndarray
    rho: float = 1.0
    dt: float = 1e-3

    @classmethod
    def from_case(cls, case, types, u, v, w, p=None) -> "MACGrid":
        g = case.grid
        p = np.zeros(g.cells) if p is None else np.ascontiguousarray(p, dtype=np.float64).reshape(-1).copy()
        return cls(g, np.ascontiguousarray(types, dtype=np.uint8).reshape(-1),
                   np.ascontiguousarray(u, dtype=np.float64).reshape(-1).copy(),
                   np.ascontiguousarray(v, dtype=np.float64).reshape(-1).copy(),
                   np.ascontiguousarray(w, dtype=np.float64).reshape(-1).copy(), p, case.rho, case.dt)


class PressureSolver:
    """One pressure system on one GPU (the reference keeps one static system per dimension)."""

    def __init__(self, precision: str = "mixed", device: int = 0, stream: Optional[int] = None, **options):
        self.lib = capi.load()
        prec = {"mixed": capi.PRECISION_MIXED, "fp64": capi.PRECISION_FP64}[precision]
        self.opts = capi.default_options(device=device, precision=prec, **options)
        if stream is not None:
            self.opts.stream = ctypes.c_void_p(stream)
        self.ctx = ctypes.c_void_p()
        self._tables = None
        self.grid: Optional[MACGrid] = None
        self.last: Optional[capi.Result] = None
        self.projected = False
        self.scheme = capi.SCHEME_CHORIN
        self.warm_start = False

    # ---- life cycle (PressureSolver3D.h:52-54) ----
    def InitializePressureSolver(self, grid: MACGrid, scheme: int = capi.SCHEME_CHORIN, warm_start: bool = False):
        """scheme: SCHEME_CHORIN or SCHEME_INCREMENTAL (SYSTEM.scheme); warm_start: Chorin solves start from the
        previous pressure (PRESSURE_SETTINGS.warmStart, honoured on uniform grids as WarmStartEnabled)."""
        if scheme not in (capi.SCHEME_CHORIN, capi.SCHEME_INCREMENTAL):
            raise capi.NBError(capi.NB_BAD_INPUT, "unknown scheme %r" % (scheme,))
        self.scheme = scheme
        self.warm_start = bool(warm_start)
        if not self.ctx:
            capi.check(self.lib.nereus_b200_create(ctypes.byref(self.ctx), ctypes.byref(self.opts)))
        self.EnsureSystem(grid)

    def EnsureSystem(self, grid: MACGrid):
        """Rebuilds the hierarchy only when the layout changed (PressureLayoutChanged, PressureSettings.h:300-303);
        the library compares the cell-type bytes itself."""
        g = grid.grid
        widths = [np.ascontiguousarray(w) for w in g.width_tables()]
        gaps = [np.ascontiguousarray(x) for x in g.gap_tables()]
        self._tables = (widths, gaps, np.ascontiguousarray(grid.types, dtype=np.uint8))
        W = (capi._dp * 3)(*[capi.ptr(a) for a in widths])
        G = (capi._dp * 3)(*[capi.ptr(a) for a in gaps])
        capi.check(self.lib.nereus_b200_set_layout(self.ctx, g.dim, g.Nx, g.Ny, g.Nz,
                                                   capi.ptr(self._tables[2], capi._u8), W, G,
                                                   int(g.nonuniform), g.dh))
        self.grid = grid

    def ReleasePressureSolver(self):
        self.DestroyPressureSolver()

    def DestroyPressureSolver(self):
        if self.ctx:
            self.lib.nereus_b200_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()
        self.grid = None

    def __del__(self):
        try:
            self.DestroyPressureSolver()
        except Exception:
            pass

    # ---- the pressure step (SolveChorin / SolvePressure, PressureSolver3D.h:57-60) ----
    def SolvePressure(self, grid: MACGrid, tol: float = 1e-8, needs_compat: bool = False,
                      grid_ant: Optional[MACGrid] = None) -> capi.Result:
        """Pressure step + projection of ``grid`` in place, in the scheme chosen at initialisation. ``grid_ant``
        is the previous step's state (the reference's gridAnt): its pressure is p^n of the incremental scheme
        (required there) and the Chorin warm start's guess. Returns the solve's report; raises on bad input or a
        device error; a solve that hits its caps returns with status NOT_CONVERGED (the reference warns once)."""
        if self.grid is None or grid.grid is not self.grid.grid or not np.array_equal(grid.types, self._tables[2]):
            self.InitializePressureSolver(grid, self.scheme, self.warm_start) if not self.ctx else \
                self.EnsureSystem(grid)
        r = capi.Result()
        g = grid.grid
        w = grid.w if g.dim == 3 else np.zeros(1)
        incremental = self.scheme == capi.SCHEME_INCREMENTAL
        if incremental and grid_ant is None:
            raise capi.NBError(capi.NB_BAD_INPUT, "the incremental scheme needs the previous step's grid")
        if incremental or (self.warm_start and grid_ant is not None):
            p_prev = np.ascontiguousarray(grid_ant.p, dtype=np.float64)
            st = self.lib.nereus_b200_project_ex(self.ctx, capi.ptr(grid.u), capi.ptr(grid.v), capi.ptr(w),
                                                 capi.ptr(grid.p), capi.ptr(p_prev), grid.rho, grid.dt,
                                                 self.scheme, int(needs_compat), int(self.warm_start), tol,
                                                 ctypes.byref(r))
        else:
            st = self.lib.nereus_b200_project(self.ctx, capi.ptr(grid.u), capi.ptr(grid.v), capi.ptr(w),
                                              capi.ptr(grid.p), grid.rho, grid.dt, capi.SCHEME_CHORIN,
                                              int(needs_compat), tol, ctypes.byref(r))
        capi.check(st, allow=(capi.NB_OK, capi.NB_NOT_CONVERGED))
        self.last = r
        self.projected = True
        return r

    def SolveChorin(self, grid: MACGrid, tol: float = 1e-8, needs_compat: bool = False,
                    grid_ant: Optional[MACGrid] = None) -> capi.Result:
        """SolveChorin (PressureSolver3D.h:57): the Chorin step whatever the initialised scheme."""
        keep, self.scheme = self.scheme, capi.SCHEME_CHORIN
        try:
            return self.SolvePressure(grid, tol, needs_compat, grid_ant)
        finally:
            self.scheme = keep

    def SolveIncremental(self, grid_ant: MACGrid, grid: MACGrid, tol: float = 1e-8,
                         needs_compat: bool = False) -> capi.Result:
        """SolveIncremental + Project (PressureSolver3D.h:58,71): phi = p^{n+1} - p^n, the velocity corrected with
        grad phi, p = p^n + phi levelled."""
        keep, self.scheme = self.scheme, capi.SCHEME_INCREMENTAL
        try:
            return self.SolvePressure(grid, tol, needs_compat, grid_ant)
        finally:
            self.scheme = keep

    def ProjectPressure(self, grid: MACGrid) -> bool:
        """The velocity correction already ran inside SolvePressure; True when it did for this grid."""
        done = self.projected
        self.projected = False
        return done

    def SolveLaplacian(self, grid: MACGrid, f: np.ndarray, tol: float = 1e-12):
        """L x = f on the unknowns (PressureSolver3D.h:62-64): (False, None) when f's size is not SystemSize()."""
        if self.grid is None:
            self.InitializePressureSolver(grid)
        n = self.SystemSize()
        f = np.ascontiguousarray(f, dtype=np.float64)
        if n == 0 or f.shape[0] != n:
            return False, None
        x = np.zeros(n)
        r = capi.Result()
        st = self.lib.nereus_b200_solve_laplacian(self.ctx, capi.ptr(f), capi.ptr(x), tol, ctypes.byref(r))
        capi.check(st, allow=(capi.NB_OK, capi.NB_NOT_CONVERGED))
        self.last = r
        return True, x

    # ---- queries (PressureSolver3D.h:66-68, 75) ----
    def SystemSize(self) -> int:
        return self.lib.nereus_b200_system_size(self.ctx) if self.ctx else 0

    def LastIterations(self) -> int:
        return self.lib.nereus_b200_last_iterations(self.ctx) if self.ctx else 0

    def IDP(self) -> np.ndarray:
        idp = np.zeros(self.grid.grid.cells, dtype=np.int32)
        capi.check(self.lib.nereus_b200_get_idp(self.ctx, capi.ptr(idp, capi._ip)))
        return idp

    def GetIDP(self, i: int, j: int, k: int = 0) -> int:
        g = self.grid.grid
        return int(self.IDP()[(i * g.Nx + j) * g.Nz + k])

    # ---- what the parity tests read ----
    def ExportMatrix(self):
        n = self.SystemSize()
        g = self.grid.grid
        cap = max(n, 1) * (7 if g.dim == 3 else 5)
        rowptr = np.zeros(n + 1, dtype=np.int32)
        col = np.zeros(cap, dtype=np.int32)
        val = np.zeros(cap, dtype=np.float64)
        nnz, sing = ctypes.c_int(0), ctypes.c_int(0)
        capi.check(self.lib.nereus_b200_export_matrix(self.ctx, capi.ptr(rowptr, capi._ip), capi.ptr(col, capi._ip),
                                                      capi.ptr(val), ctypes.byref(nnz), ctypes.byref(sing)))
        return rowptr, col[: nnz.value].copy(), val[: nnz.value].copy(), bool(sing.value)

    def Rhs(self, grid: MACGrid) -> np.ndarray:
        n = self.SystemSize()
        b = np.zeros(max(n, 1))
        w = grid.w if grid.grid.dim == 3 else np.zeros(1)
        capi.check(self.lib.nereus_b200_rhs(self.ctx, capi.ptr(grid.u), capi.ptr(grid.v), capi.ptr(w),
                                            capi.ptr(grid.p), grid.rho, grid.dt, capi.ptr(b)))
        return b[:n]
