"""The boundary-condition replay of a MAC grid on the device: MAC::EnforceVelocityBC and MAC::EnforcePressureBC
(src/MAC.cpp:811-865) from the lists MAC::BuildBoundaryLists made (src/MAC.cpp:613-1090), through
nereus_b200_bc_create / _enforce_velocity / _enforce_pressure. Fields are device arrays (torch CUDA tensors or raw
device pointers); the calls queue work on a stream and return."""
from __future__ import annotations

import ctypes

import numpy as np

from . import capi

LIST_KEYS = ("solid0", "solid1", "solid2", "presc_comp", "presc_index", "copy_comp", "copy_dst", "copy_src",
             "ring_dst", "ring_kind", "ring_src", "inlet_comp", "inlet_index", "inlet_area", "inlet_sign",
             "outflow_comp", "outflow_index", "outflow_outer", "outflow_area", "outflow_sign")


def _ptr(x):
    if x is None:
        return None
    if hasattr(x, "cuda_stream"):
        return ctypes.c_void_p(x.cuda_stream)
    if hasattr(x, "data_ptr"):
        return ctypes.c_void_p(x.data_ptr())
    return ctypes.c_void_p(int(x))


def make_lists(lists, dim: int, Nx: int, Ny: int, Nz: int):
    """nb_bc_lists over ``lists`` (the names of LIST_KEYS mapped to arrays); returns the struct and the arrays it
    points into, which must outlive it."""
    i32 = lambda k: np.ascontiguousarray(lists[k], dtype=np.int32)
    f64 = lambda k: np.ascontiguousarray(lists[k], dtype=np.float64)
    K = {k: (f64(k) if k.endswith(("_area", "_sign")) else i32(k)) for k in LIST_KEYS}
    ip = lambda k: K[k].ctypes.data_as(capi._i32p)
    dp = lambda k: K[k].ctypes.data_as(capi._dp)
    L = capi.BcLists()
    L.dim, L.Nx, L.Ny, L.Nz = dim, Nx, Ny, Nz if dim == 3 else 1
    for c in range(3):
        L.solid[c] = ip("solid%d" % c)
        L.nsolid[c] = len(K["solid%d" % c])
    L.presc_comp, L.presc_index, L.npresc = ip("presc_comp"), ip("presc_index"), len(K["presc_comp"])
    L.copy_comp, L.copy_dst, L.copy_src, L.ncopy = ip("copy_comp"), ip("copy_dst"), ip("copy_src"), len(K["copy_comp"])
    L.ring_dst, L.ring_kind, L.ring_src, L.nring = ip("ring_dst"), ip("ring_kind"), ip("ring_src"), len(K["ring_dst"])
    L.inlet_comp, L.inlet_index, L.inlet_area, L.inlet_sign = (ip("inlet_comp"), ip("inlet_index"), dp("inlet_area"),
                                                               dp("inlet_sign"))
    L.ninlet = len(K["inlet_comp"])
    L.outflow_comp, L.outflow_index, L.outflow_outer = ip("outflow_comp"), ip("outflow_index"), ip("outflow_outer")
    L.outflow_area, L.outflow_sign, L.noutflow = dp("outflow_area"), dp("outflow_sign"), len(K["outflow_comp"])
    return L, K


def plan_levels(lists, dim: int, Nx: int, Ny: int, Nz: int):
    """The level each entry is replayed in (nereus_b200_bc_plan, host only): velocity levels for the solid faces of
    u, v, w, the prescribed entries and the copies, in that order; pressure levels for the ring entries."""
    lib = capi.load()
    L, K = make_lists(lists, dim, Nx, Ny, Nz)
    nv = sum(len(K["solid%d" % c]) for c in range(3)) + len(K["presc_comp"]) + len(K["copy_comp"])
    vel = np.zeros(nv, dtype=np.int32)
    pres = np.zeros(len(K["ring_dst"]), dtype=np.int32)
    a, b = ctypes.c_int(), ctypes.c_int()
    capi.check(lib.nereus_b200_bc_plan(ctypes.byref(L), ctypes.c_void_p(vel.ctypes.data),
                                       ctypes.c_void_p(pres.ctypes.data), ctypes.byref(a), ctypes.byref(b)))
    return vel, pres, a.value, b.value


class BoundaryReplay:
    """One grid's boundary lists on one device. ``lists`` maps the names of LIST_KEYS to arrays (a bc_* fixture,
    or the arrays a host MAC exports); dim and Nx, Ny, Nz (ring included) give the field sizes the indices are
    checked against."""

    def __init__(self, lists, dim: int, Nx: int, Ny: int, Nz: int, device: int = 0):
        self.lib = capi.load()
        L, self._keep = make_lists(lists, dim, Nx, Ny, Nz)
        self.dim = dim
        self.handle = ctypes.c_void_p()
        capi.check(self.lib.nereus_b200_bc_create(device, ctypes.byref(L), ctypes.byref(self.handle)))

    def levels(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        capi.check(self.lib.nereus_b200_bc_levels(self.handle, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def EnforceVelocityBC(self, u, v, w, presc_values=None, stream=None):
        """presc_values: device array of the boundary velocity function's components at the prescribed entries,
        or None when the scene has no boundary velocity function."""
        capi.check(self.lib.nereus_b200_bc_enforce_velocity(self.handle, _ptr(u), _ptr(v), _ptr(w),
                                                            _ptr(presc_values), _ptr(stream)))

    def EnforcePressureBC(self, p, ring_values=None, stream=None):
        """ring_values: device array read at the ring's prescribed (kind 1) entries; None writes 0 there."""
        capi.check(self.lib.nereus_b200_bc_enforce_pressure(self.handle, _ptr(p), _ptr(ring_values), _ptr(stream)))

    def close(self):
        if self.handle:
            self.lib.nereus_b200_bc_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
