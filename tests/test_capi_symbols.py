"""The C ABI library (CPU side): it builds for sm_100a, loads, exports every entry point include/nereus_b200.h
declares with the ctypes signature the bindings use, and refuses to run without a GPU instead of falling back."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, cuda_ok
from nereus_cfd_b200 import build, capi

HEADER = os.path.join(ROOT, "include", "nereus_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nereus_b200_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return capi.load()


def test_header_declares_the_backend_entry_points():
    """The calls a NEREUS pressure backend needs: context, layout, the projection step and SolveLaplacian."""
    syms = declared_symbols()
    for s in ["nereus_b200_create", "nereus_b200_destroy", "nereus_b200_set_layout", "nereus_b200_project",
              "nereus_b200_solve_laplacian"]:
        assert s in syms


def test_every_declared_symbol_is_exported(lib):
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
        assert s in capi.SIGNATURES, "no ctypes signature for %s" % s
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\b(nereus_b200_\w+)\b", out))
    assert set(syms) <= exported


def test_built_for_sm100a_only():
    flags = " ".join(build.ARCH)
    assert "arch=compute_100a,code=sm_100a" in flags
    assert len(re.findall(r"-gencode", flags)) == 1


def test_default_options(lib):
    o = capi.default_options()
    assert o.precision == capi.PRECISION_MIXED
    assert o.max_iters > 0 and o.max_outer > 0 and 0 < o.inner_tol < 1
    assert o.pre_sweeps >= 1 and o.post_sweeps >= 1 and o.max_levels >= 1


@pytest.mark.skipif(cuda_ok(), reason="checks the no-GPU behaviour")
def test_no_device_is_an_error_not_a_fallback(lib):
    ctx = ctypes.c_void_p()
    st = lib.nereus_b200_create(ctypes.byref(ctx), None)
    assert st == capi.NB_NO_DEVICE
    assert not ctx
    assert lib.nereus_b200_device_count() == 0


def test_null_arguments_are_bad_input(lib):
    assert lib.nereus_b200_create(None, None) == capi.NB_BAD_INPUT
    assert lib.nereus_b200_project(None, None, None, None, None, 1.0, 1.0, 0, 0, 1e-8, None) == capi.NB_BAD_INPUT
    assert lib.nereus_b200_system_size(None) == 0
    lib.nereus_b200_destroy(None)  # a no-op


def test_relabel_checks_its_arguments_before_the_device(lib):
    """nereus_b200_update_fluid_cells refuses bad sizes and pointers before it looks for a device."""
    t = np.zeros(27, dtype=np.uint8)
    xyz = np.zeros((2, 3))
    px = ctypes.c_void_p(xyz.ctypes.data)
    args = lambda **kw: dict(dict(dim=3, N=3, t=capi.ptr(t, capi._u8), px=px, count=2, stride=3), **kw)

    def call(a):
        return lib.nereus_b200_update_fluid_cells(a["dim"], a["N"], a["N"], a["N"], 0.0, 0.0, 0.0, 1.0, a["px"],
                                                  a["px"], a["px"], a["count"], a["stride"], a["t"], None)
    assert call(args(t=None)) == capi.NB_BAD_INPUT
    assert call(args(dim=4)) == capi.NB_BAD_INPUT
    assert call(args(N=0)) == capi.NB_BAD_INPUT
    assert call(args(count=-1)) == capi.NB_BAD_INPUT
    assert call(args(stride=0)) == capi.NB_BAD_INPUT
    assert call(args(px=None)) == capi.NB_BAD_INPUT
    if not cuda_ok():
        assert call(args()) == capi.NB_NO_DEVICE
        sb = lib.nereus_b200_update_fluid_cells_scratch_bytes(3, 10, 10, 10)
        assert sb == 16 + 4 * 8 ** 3


@pytest.mark.skipif(cuda_ok(), reason="checks the no-GPU behaviour")
def test_cpp_host_side_errors_without_a_device(lib, tmp_path):
    """include/nereus_b200_solver.hpp's UpdateFluidCells and BoundaryReplay: NB_BAD_INPUT for bad arguments,
    NB_NO_DEVICE (an exception, not a host fallback) for a good call without a GPU."""
    exe = str(tmp_path / "shim_errors")
    libdir = os.path.dirname(capi.LIB_PATH)
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "shim_errors.cpp"), "-o", exe, "-L" + libdir,
                           "-lnereus_b200", "-Wl,-rpath," + libdir])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr


def test_relabel_wrapper_wants_a_coordinate_per_axis(lib):
    """capi.update_fluid_cells reads x, y (, z) from each row: a 3D call with two columns is refused in Python."""
    from nereus_cfd_b200 import workloads as W

    g = W.flip_tank_3d(n=4, seed=1).grid
    with pytest.raises(ValueError):
        capi.update_fluid_cells(g, np.zeros(g.cells, dtype=np.uint8), np.zeros((3, 2)), [0.0, 0.0, 0.0])
