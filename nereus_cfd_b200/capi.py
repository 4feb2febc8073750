"""ctypes binding of the B200 library's C ABI (include/nereus_b200.h).

The library is ``nereus_cfd_b200/libnereus_b200.so``, built in-tree by ``nereus_cfd_b200.build``. Loading fails with
an error when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnereus_b200.so")

NB_OK, NB_NOT_CONVERGED, NB_BAD_INPUT, NB_OUT_OF_MEMORY, NB_DEVICE_ERROR, NB_NO_DEVICE, NB_BUSY = range(7)
STATUS_NAMES = {0: "OK", 1: "NOT_CONVERGED", 2: "BAD_INPUT", 3: "OUT_OF_MEMORY", 4: "DEVICE_ERROR",
                5: "NO_DEVICE", 6: "BUSY"}
PRECISION_FP64, PRECISION_MIXED = 0, 1
SCHEME_CHORIN, SCHEME_INCREMENTAL = 0, 1

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_u8 = ctypes.POINTER(ctypes.c_uint8)


class Options(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("precision", ctypes.c_int), ("max_iters", ctypes.c_int),
                ("max_outer", ctypes.c_int), ("inner_tol", ctypes.c_double), ("pre_sweeps", ctypes.c_int),
                ("post_sweeps", ctypes.c_int), ("coarse_sweeps", ctypes.c_int), ("max_levels", ctypes.c_int),
                ("stream", ctypes.c_void_p), ("use_graphs", ctypes.c_int), ("transfer_kernels", ctypes.c_int),
                ("pair_kernels", ctypes.c_int), ("tail_cells", ctypes.c_int), ("stretched_sweeps", ctypes.c_int),
                ("autotune", ctypes.c_int), ("skip_idle_tiles", ctypes.c_int),
                ("x_groups", ctypes.c_int)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("n", ctypes.c_int), ("singular", ctypes.c_int),
                ("iters_outer", ctypes.c_int), ("iters_inner", ctypes.c_int), ("levels", ctypes.c_int),
                ("b_norm", ctypes.c_double), ("rel_res", ctypes.c_double), ("max_div", ctypes.c_double),
                ("seconds", ctypes.c_double), ("latency_ms", ctypes.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class ServerOptions(ctypes.Structure):
    _fields_ = [("n_devices", ctypes.c_int), ("devices", ctypes.POINTER(ctypes.c_int)),
                ("slots_per_device", ctypes.c_int), ("hbm_budget_gb", ctypes.c_double), ("solver", Options)]


class Request(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int),
                ("cell_types", ctypes.POINTER(ctypes.c_uint8)), ("width", ctypes.POINTER(ctypes.c_double) * 3),
                ("gap", ctypes.POINTER(ctypes.c_double) * 3), ("non_uniform", ctypes.c_int), ("dh", ctypes.c_double),
                ("u", ctypes.POINTER(ctypes.c_double)), ("v", ctypes.POINTER(ctypes.c_double)),
                ("w", ctypes.POINTER(ctypes.c_double)), ("p", ctypes.POINTER(ctypes.c_double)),
                ("p_prev", ctypes.POINTER(ctypes.c_double)), ("scheme", ctypes.c_int), ("needs_compat", ctypes.c_int),
                ("warm_start", ctypes.c_int), ("rho", ctypes.c_double), ("dt", ctypes.c_double),
                ("tol", ctypes.c_double), ("fields_on_device", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong), ("failed", ctypes.c_longlong),
                ("queued", ctypes.c_longlong), ("running", ctypes.c_longlong), ("seconds", ctypes.c_double),
                ("solves_per_s", ctypes.c_double), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("admitted_gb", ctypes.c_double),
                ("device_completed", ctypes.c_longlong * 8), ("layout_s", ctypes.c_double),
                ("project_s", ctypes.c_double)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f != "device_completed"}
        d["device_completed"] = list(self.device_completed)
        return d


class Region(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("region", ctypes.c_int), ("axis", ctypes.c_int), ("invert", ctypes.c_int),
                ("p0", ctypes.c_double * 3), ("p1", ctypes.c_double * 3), ("radius", ctypes.c_double)]


class SceneStruct(ctypes.Structure):
    _fields_ = [("face_kind", ctypes.c_int * 6), ("face_has_p", ctypes.c_int * 6), ("face_order", ctypes.c_int * 6),
                ("nregions", ctypes.c_int), ("regions", Region * 16)]


class BatchItem(ctypes.Structure):
    """nb_batch_item: one request of a batched step (device fields of its slot)."""

    _fields_ = [("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("w", ctypes.c_void_p), ("p", ctypes.c_void_p),
                ("rho", ctypes.c_double), ("dt", ctypes.c_double), ("needs_compat", ctypes.c_int),
                ("tol", ctypes.c_double)]


BATCH_MAX_LEVELS = 16
BATCH_KINDS = ["first", "half", "residual", "restrict", "prolong"]


class BatchInfo(ctypes.Structure):
    _fields_ = [("capacity", ctypes.c_int), ("levels", ctypes.c_int), ("tail_start", ctypes.c_int),
                ("loop_launches", ctypes.c_longlong), ("tune_ms", ctypes.c_double),
                ("march", (ctypes.c_int * 5) * BATCH_MAX_LEVELS), ("restrict_mode", ctypes.c_int * BATCH_MAX_LEVELS)]

    def as_dict(self):
        n = max(0, self.tail_start)
        return {"capacity": self.capacity, "levels": self.levels, "tail_start": self.tail_start,
                "loop_launches": self.loop_launches, "tune_ms": round(self.tune_ms, 3),
                "march": [dict(zip(BATCH_KINDS, list(self.march[l]))) for l in range(n)],
                "restrict_mode": [self.restrict_mode[l] for l in range(n)]}


# Every exported symbol of include/nereus_b200.h with its ctypes signature.
_i32p = ctypes.POINTER(ctypes.c_int32)


class BcLists(ctypes.Structure):
    """nb_bc_lists (include/nereus_b200.h): the MAC's boundary lists for nereus_b200_bc_create."""

    _fields_ = [("dim", ctypes.c_int), ("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int),
                ("solid", _i32p * 3), ("nsolid", ctypes.c_int32 * 3),
                ("presc_comp", _i32p), ("presc_index", _i32p), ("npresc", ctypes.c_int32),
                ("copy_comp", _i32p), ("copy_dst", _i32p), ("copy_src", _i32p), ("ncopy", ctypes.c_int32),
                ("ring_dst", _i32p), ("ring_kind", _i32p), ("ring_src", _i32p), ("nring", ctypes.c_int32),
                ("inlet_comp", _i32p), ("inlet_index", _i32p), ("inlet_area", _dp), ("inlet_sign", _dp),
                ("ninlet", ctypes.c_int32),
                ("outflow_comp", _i32p), ("outflow_index", _i32p), ("outflow_outer", _i32p), ("outflow_area", _dp),
                ("outflow_sign", _dp), ("noutflow", ctypes.c_int32)]


SIGNATURES = {
    "nereus_b200_default_options": (None, [ctypes.POINTER(Options)]),
    "nereus_b200_last_error": (ctypes.c_char_p, []),
    "nereus_b200_device_count": (ctypes.c_int, []),
    "nereus_b200_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(Options)]),
    "nereus_b200_destroy": (None, [ctypes.c_void_p]),
    "nereus_b200_set_layout": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, _u8, _dp * 3, _dp * 3, ctypes.c_int, ctypes.c_double]),
    "nereus_b200_project": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.POINTER(Result)]),
    "nereus_b200_project_ex": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_double, ctypes.POINTER(Result)]),
    "nereus_b200_project_device_ex": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                     ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                                     ctypes.c_int, ctypes.c_double, ctypes.POINTER(Result)]),
    "nereus_b200_solve_pressure": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, _dp, ctypes.c_double,
                                                  ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                  ctypes.POINTER(Result)]),
    "nereus_b200_project_velocity": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, _dp, ctypes.c_double,
                                                    ctypes.c_double]),
    "nereus_b200_project_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                                  ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                                  ctypes.POINTER(Result)]),
    "nereus_b200_solve_laplacian": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, ctypes.c_double,
                                                   ctypes.POINTER(Result)]),
    "nereus_b200_system_size": (ctypes.c_int, [ctypes.c_void_p]),
    "nereus_b200_last_iterations": (ctypes.c_int, [ctypes.c_void_p]),
    "nereus_b200_get_idp": (ctypes.c_int, [ctypes.c_void_p, _ip]),
    "nereus_b200_export_matrix": (ctypes.c_int, [ctypes.c_void_p, _ip, _ip, _dp, ctypes.POINTER(ctypes.c_int),
                                                 ctypes.POINTER(ctypes.c_int)]),
    "nereus_b200_rhs": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double,
                                       _dp]),
    "nereus_b200_label_cells": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp,
                                               _dp, ctypes.POINTER(SceneStruct), _u8]),
    "nereus_b200_profile_enable": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint]),
    "nereus_b200_profile_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "nereus_b200_kernel_launches": (ctypes.c_longlong, []),
    "nereus_b200_default_server_options": (None, [ctypes.POINTER(ServerOptions)]),
    "nereus_b200_server_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ServerOptions)]),
    "nereus_b200_server_destroy": (None, [ctypes.c_void_p]),
    "nereus_b200_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Request),
                                          ctypes.POINTER(ctypes.c_uint64)]),
    "nereus_b200_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Result)]),
    "nereus_b200_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double,
                                        ctypes.POINTER(Result)]),
    "nereus_b200_server_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerStats)]),
    "nereus_b200_server_reset_stats": (ctypes.c_int, [ctypes.c_void_p]),
    "nereus_b200_request_bytes": (ctypes.c_double, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_int]),
    "nereus_b200_plan": (ctypes.c_int, [_dp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "nereus_b200_number_unknowns_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                           ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                           ctypes.c_void_p, ctypes.c_void_p]),
    "nereus_b200_update_fluid_cells": (ctypes.c_int, [ctypes.c_int] * 4 + [ctypes.c_double] * 4 +
                                       [ctypes.c_void_p] * 3 + [ctypes.c_int64, ctypes.c_int64, _u8,
                                                                ctypes.POINTER(ctypes.c_int64)]),
    "nereus_b200_update_fluid_cells_scratch_bytes": (ctypes.c_size_t, [ctypes.c_int] * 4),
    "nereus_b200_bc_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(BcLists), ctypes.POINTER(ctypes.c_void_p)]),
    "nereus_b200_bc_enforce_velocity": (ctypes.c_int, [ctypes.c_void_p] * 6),
    "nereus_b200_bc_enforce_pressure": (ctypes.c_int, [ctypes.c_void_p] * 4),
    "nereus_b200_bc_levels": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int)]),
    "nereus_b200_bc_destroy": (None, [ctypes.c_void_p]),
    "nereus_b200_bc_plan": (ctypes.c_int, [ctypes.POINTER(BcLists), ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "nereus_b200_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(Options),
                                                ctypes.c_int]),
    "nereus_b200_batch_destroy": (None, [ctypes.c_void_p]),
    "nereus_b200_batch_set_layout": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_int, ctypes.c_int, _u8, _dp * 3, _dp * 3, ctypes.c_int,
                                                    ctypes.c_double]),
    "nereus_b200_batch_project_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(BatchItem),
                                                        ctypes.POINTER(Result)]),
    "nereus_b200_batch_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchInfo)]),
    "nereus_b200_tune_choose": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int]),
    "nereus_b200_x_groups": (ctypes.c_int, [_dp, ctypes.c_int, ctypes.c_double, _ip]),
    "nereus_b200_x_maps": (ctypes.c_int, [_dp, ctypes.c_int, ctypes.c_double, _ip, _ip]),
    "nereus_b200_tune_key": (ctypes.c_int, [ctypes.c_int] * 6 + [ctypes.c_char_p, ctypes.c_int]),
    "nereus_b200_tune_cache_dump": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int]),
    "nereus_b200_tune_cache_load": (ctypes.c_int, [ctypes.c_char_p]),
    "nereus_b200_tune_cache_clear": (None, []),
    "nereus_b200_update_fluid_cells_device": (ctypes.c_int, [ctypes.c_int] * 5 + [ctypes.c_double] * 4 +
                                              [ctypes.c_void_p] * 3 + [ctypes.c_int64, ctypes.c_int64] +
                                              [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                               ctypes.c_void_p]),
}

# kernel ids of nereus_b200_profile_* (include/nereus_b200.h)
KERNEL_NAMES = ["smooth0", "residual0", "restrict0", "prolong0", "p_apply", "xr_update", "dot", "refine64", "rhs",
                "project", "coarse_levels"]


def profile_read(lib, ctx):
    """{kernel name: (launches, total ms, algorithmic bytes per launch)} of the profiled kernels."""
    out = {}
    for k, name in enumerate(KERNEL_NAMES):
        n, ms, by = ctypes.c_int(0), ctypes.c_double(0.0), ctypes.c_double(0.0)
        check(lib.nereus_b200_profile_read(ctx, k, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(by)))
        if n.value:
            out[name] = (n.value, ms.value, by.value)
    return out

_LIB = None


def load(path: str = LIB_PATH):
    """The loaded library with every signature declared. Raises when the shared object is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError("%s is not built: run `python -m nereus_cfd_b200.build` (no CPU fallback exists)" % path)
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


class NBError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), msg))
        self.status = status


def check(status: int, allow=(NB_OK,)):
    if status not in allow:
        raise NBError(status, load().nereus_b200_last_error().decode(errors="replace"))
    return status


def ptr(a: np.ndarray, t=_dp):
    return a.ctypes.data_as(t)


def default_options(**kw) -> Options:
    o = Options()
    load().nereus_b200_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def scene_struct(scene) -> SceneStruct:
    s = SceneStruct()
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


def update_fluid_cells(grid, types, xyz, origin, dh=None):
    """FLIP{2,3}D::UpdateFluidCells on the device from host arrays (nereus_b200_update_fluid_cells): returns the new
    cell types and the number of particles skipped as outside the labels. xyz: (count, 3) float64 positions, or any
    float64 array whose rows start with x, y, z (the reference's 7-double Particle rows included); origin:
    FacePos(X|Y|Z, 0)."""
    out = np.ascontiguousarray(types, dtype=np.uint8).reshape(-1).copy()
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    xyz = xyz.reshape(xyz.shape[0], -1) if xyz.size else np.zeros((0, 3))
    count, stride = xyz.shape
    if count and stride < grid.dim:
        raise ValueError("positions need x, y%s in each row" % (", z" if grid.dim == 3 else ""))
    base = xyz.ctypes.data
    pz = ctypes.c_void_p(base + 16) if grid.dim == 3 else None
    skipped = ctypes.c_int64(0)
    oz = origin[2] if len(origin) > 2 else 0.0
    check(load().nereus_b200_update_fluid_cells(
        grid.dim, grid.Nx, grid.Ny, grid.Nz if grid.dim == 3 else 1, origin[0], origin[1], oz,
        grid.dh if dh is None else dh, ctypes.c_void_p(base), ctypes.c_void_p(base + 8), pz, count, stride,
        ptr(out, _u8), ctypes.byref(skipped)))
    return out, int(skipped.value)


def label_cells(grid, scene) -> np.ndarray:
    """Scene::CellTypeAt for every cell, on the device."""
    cx, cy, cz = [np.ascontiguousarray(c, dtype=np.float64) for c in grid.sample_coords(scene.at_centre)]
    out = np.zeros(grid.cells, dtype=np.uint8)
    s = scene_struct(scene)
    check(load().nereus_b200_label_cells(grid.dim, grid.Nx, grid.Ny, grid.Nz, ptr(cx), ptr(cy), ptr(cz),
                                         ctypes.byref(s), ptr(out, _u8)))
    return out
