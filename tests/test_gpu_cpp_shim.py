"""The C++ host side (include/nereus_b200_solver.hpp): a program built against the shim and the library projects a
case exactly as the Python mirror does (same library, same launch sequence: bit-identical results)."""
import os
import struct
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, load_golden
from nereus_cfd_b200 import capi
from nereus_cfd_b200.pressure import MACGrid, PressureSolver

SRC = os.path.join(ROOT, "tests", "cpp", "shim_project.cpp")


def build_shim(out_dir):
    exe = os.path.join(out_dir, "shim_project")
    cmd = ["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L" + os.path.dirname(capi.LIB_PATH), "-lnereus_b200", "-Wl,-rpath," + os.path.dirname(capi.LIB_PATH)]
    subprocess.check_call(cmd)
    return exe


def test_shim_compiles(tmp_path):
    """Compiles and links on any machine with the library built (no GPU needed)."""
    capi.load()
    assert os.path.exists(build_shim(str(tmp_path)))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sphere_outlet_3d_12", "channel_2d_stretched_24x12"])
def test_shim_matches_python_mirror(nb, tmp_path, name):
    case, meta, z = load_golden(name)
    g = case.grid
    exe = build_shim(str(tmp_path))
    tol = 1e-10
    cpath, rpath = os.path.join(str(tmp_path), "case.bin"), os.path.join(str(tmp_path), "res.bin")
    with open(cpath, "wb") as f:
        f.write(struct.pack("<5i", g.dim, g.Nx, g.Ny, g.Nz, int(g.nonuniform)))
        f.write(struct.pack("<4d", g.dh, meta["rho"], meta["dt"], tol))
        f.write(z["types"].astype(np.uint8).tobytes())
        for t in g.width_tables():
            f.write(t.astype("<f8").tobytes())
        for t in g.gap_tables():
            f.write(t.astype("<f8").tobytes())
        for a in (z["u"], z["v"], z["w"], z["p_in"]):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
    subprocess.check_call([exe, cpath, rpath])
    data = open(rpath, "rb").read()
    status, n, iters = struct.unpack_from("<3i", data, 0)
    (rel,) = struct.unpack_from("<d", data, 12)
    off = 20
    p = np.frombuffer(data, "<f8", g.cells, off)
    off += 8 * g.cells
    u = np.frombuffer(data, "<f8", z["u"].size, off)
    assert status == capi.NB_OK and n == meta["n"] and rel <= tol
    s = PressureSolver("mixed")
    m = MACGrid(g, z["types"].copy(), z["u"].copy(), z["v"].copy(), z["w"].copy(), z["p_in"].copy(), meta["rho"],
                meta["dt"])
    r = s.SolvePressure(m, tol=tol)
    assert r.iters_inner == iters
    assert np.array_equal(m.p, p) and np.array_equal(m.u, u)
    s.DestroyPressureSolver()
