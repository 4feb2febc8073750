"""ORACLE / TEST INFRASTRUCTURE ONLY: runs the reference's own pressure path (``oracle/_ref/ref_harness``, compiled
from the reference sources by ``oracle/Makefile``) on one case and reads back what it computed.

The case file format is documented at the top of ``oracle/ref_harness.cpp``.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(_HERE, "_ref", "ref_harness")
SOLVER_CG, SOLVER_AMG, SOLVER_BICGSTAB = 0, 1, 2


def available() -> bool:
    return os.path.exists(HARNESS)


def build(ref_root: str = "/root/reference") -> bool:
    """Compiles the harness when the reference sources are present; True when the binary exists afterwards."""
    if os.path.isdir(ref_root):
        subprocess.check_call(["make", "-s", "-C", _HERE, "ref", "REF=" + ref_root, "-j8"])
    return available()


@dataclass
class RefResult:
    Nx: int
    Ny: int
    Nz: int
    n: int
    iters: int
    singular: bool
    threads: int
    t_assemble: float
    t_solve_cold: float
    t_solve_warm: float
    t_project: float
    rel_res: float
    max_div: float
    dh: float
    types: np.ndarray
    idp: np.ndarray
    rowptr: np.ndarray
    col: np.ndarray
    val: np.ndarray
    b_raw: np.ndarray
    b: np.ndarray
    x: np.ndarray
    p: np.ndarray
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    width: list
    gap: list
    centre: list
    t_each: np.ndarray  # wall time of each warm repeat
    ref_norm: float = 0.0  # IncrementReferenceNorm (incremental scheme)
    p_final: np.ndarray = None  # the pressure after Project (schemes 1 and 2)
    origin: tuple = None  # FacePos(X|Y|Z, 0) (scheme 4)
    types_before: np.ndarray = None  # the labels UpdateFluidCells started from (scheme 4)


SCHEME_CHORIN, SCHEME_INCREMENTAL, SCHEME_CHORIN_WARM, SCHEME_EXPLICIT, SCHEME_FLIP_RELABEL = 0, 1, 2, 3, 4
SCHEME_BC_REPLAY = 5
_PREV_SCHEMES = (SCHEME_INCREMENTAL, SCHEME_CHORIN_WARM)  # the schemes that read and write a previous step


def write_case(path, case, u, v, w, label_mode=0, types=None, solver=SOLVER_CG, tol=None, max_iters=1000000,
               threads=1, repeats=0, scheme=SCHEME_CHORIN, p_prev=None, time=0.0, particles=None):
    g = case.grid
    grid_mode = 0 if not g.nonuniform else 1
    nxi, nyi = g.Nx - 2, g.Ny - 2
    nzi = g.Nz - 2 if g.dim == 3 else 0
    hdr = [g.dim, grid_mode, g.grid_size, nxi, nyi, nzi, label_mode, int(case.needs_compat), scheme, solver,
           max_iters, threads, case.method, repeats, g.Nx, g.Ny]
    with open(path, "wb") as f:
        f.write(b"NBCASE01")
        f.write(struct.pack("<16i", *hdr))
        f.write(struct.pack("<6d", *g.domain))
        f.write(struct.pack("<4d", case.rho, case.dt, case.tol if tol is None else tol, time))
        if grid_mode == 1:
            for a in range(g.dim):
                f.write(np.ascontiguousarray(g.interior_widths[a], dtype="<f8").tobytes())
        if label_mode == 0:
            text = case.scene.to_text().encode()
            f.write(struct.pack("<i", len(text)))
            f.write(text)
        else:
            f.write(np.ascontiguousarray(types, dtype=np.uint8).tobytes())
        f.write(np.ascontiguousarray(u, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(v, dtype="<f8").tobytes())
        if g.dim == 3:
            f.write(np.ascontiguousarray(w, dtype="<f8").tobytes())
        if scheme in _PREV_SCHEMES or scheme == SCHEME_BC_REPLAY:
            f.write(np.ascontiguousarray(p_prev, dtype="<f8").reshape(-1).tobytes())
        if scheme == SCHEME_FLIP_RELABEL:
            xyz = np.ascontiguousarray(particles, dtype="<f8").reshape(-1, 3)
            f.write(struct.pack("<q", xyz.shape[0]))
            f.write(xyz.tobytes())


def read_result(path, dim, scheme=SCHEME_CHORIN) -> RefResult:
    with open(path, "rb") as f:
        data = f.read()
    assert data[:8] == b"NBRES001", "bad result file"
    off = 8
    Nx, Ny, Nz, n, nnz, iters, sing, thr = struct.unpack_from("<8i", data, off)
    off += 32
    tA, tC, tW, tP, rr, md, dh, lean = struct.unpack_from("<8d", data, off)
    off += 64
    cells = Nx * Ny * Nz
    lean = lean == 1.0  # NB_REF_LEAN: no labels, numbering, matrix or right-hand sides in the file

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(data, dtype=dtype, count=count, offset=off).copy()
        off += a.nbytes
        return a

    types = take(np.uint8, 0 if lean else cells)
    idp = take("<i4", 0 if lean else cells)
    rowptr = take("<i4", 0 if lean else n + 1)
    col = take("<i4", nnz)
    val = take("<f8", nnz)
    b_raw = take("<f8", 0 if lean else n)
    b = take("<f8", 0 if lean else n)
    x = take("<f8", n)
    p = take("<f8", cells)
    u = take("<f8", (Nx + 1) * Ny * Nz)
    v = take("<f8", Nx * (Ny + 1) * Nz)
    w = take("<f8", Nx * Ny * (Nz + 1)) if dim == 3 else np.zeros(0)
    width, gap, centre = [], [], []
    for _ in range(3):
        (nw,) = struct.unpack_from("<i", data, off); off += 4
        width.append(take("<f8", nw))
        (ng,) = struct.unpack_from("<i", data, off); off += 4
        gap.append(take("<f8", ng))
        (nc,) = struct.unpack_from("<i", data, off); off += 4
        centre.append(take("<f8", nc))
    t_each = np.zeros(0)
    if off + 4 <= len(data):
        (nr,) = struct.unpack_from("<i", data, off); off += 4
        t_each = take("<f8", nr)
    ref_norm, p_final = 0.0, None
    if scheme in _PREV_SCHEMES:
        (ref_norm,) = struct.unpack_from("<d", data, off); off += 8
        p_final = take("<f8", cells)
    origin, types_before = None, None
    if scheme == SCHEME_FLIP_RELABEL:
        origin = tuple(take("<f8", 3))
        types_before = take(np.uint8, cells)
    return RefResult(Nx, Ny, Nz, n, iters, bool(sing), thr, tA, tC, tW, tP, rr, md, dh, types, idp, rowptr, col, val,
                     b_raw, b, x, p, u, v, w, width, gap, centre, t_each, ref_norm, p_final, origin, types_before)


def run(case, u, v, w, label_mode=0, types=None, solver=SOLVER_CG, tol=None, max_iters=1000000, threads=1,
        repeats=0, timeout=3600, scheme=SCHEME_CHORIN, p_prev=None, time=0.0, particles=None,
        lean=False) -> RefResult:
    """Runs the reference on ``case`` with face velocities u, v, w; labels from the scene text (label_mode 0) or
    the given ``types`` (label_mode 1). lean: the result leaves out labels, IDP, the matrix and the right-hand sides
    (empty arrays here), for large grids."""
    if not available():
        raise RuntimeError("oracle/_ref/ref_harness is not built (make -C oracle ref)")
    with tempfile.TemporaryDirectory() as td:
        cp, rp = os.path.join(td, "case.bin"), os.path.join(td, "res.bin")
        write_case(cp, case, u, v, w, label_mode, types, solver, tol, max_iters, threads, repeats, scheme, p_prev,
                   time, particles)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), NB_REF_LEAN="1" if lean else "0")
        r = subprocess.run([HARNESS, cp, rp], capture_output=True, text=True, timeout=timeout, env=env, cwd=td)
        if r.returncode != 0:
            raise RuntimeError("ref_harness failed (%d): %s %s" % (r.returncode, r.stdout[-2000:], r.stderr[-2000:]))
        return read_result(rp, case.grid.dim, scheme)


def read_bc_result(path, dim) -> dict:
    """The lists and fields of a boundary-replay run (scheme 5), as named arrays."""
    with open(path, "rb") as f:
        data = f.read()
    assert data[:8] == b"NBBC0001", "bad result file"
    off = 8
    Nx, Ny, Nz, s0, s1, s2, npresc, ncopy, nring, nin, nout = struct.unpack_from("<11i", data, off)
    off += 44

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(data, dtype=dtype, count=count, offset=off).copy()
        off += a.nbytes
        return a

    r = {"Nx": Nx, "Ny": Ny, "Nz": Nz}
    for c, n in enumerate((s0, s1, s2)):
        r["solid%d" % c] = take("<i4", n)
    r["presc_comp"], r["presc_index"], r["presc_value"] = take("<i4", npresc), take("<i4", npresc), take("<f8", npresc)
    r["copy_comp"], r["copy_dst"], r["copy_src"] = take("<i4", ncopy), take("<i4", ncopy), take("<i4", ncopy)
    r["ring_dst"], r["ring_kind"], r["ring_src"], r["ring_value"] = (take("<i4", nring), take("<i4", nring),
                                                                     take("<i4", nring), take("<f8", nring))
    for name, n in (("inlet", nin), ("outflow", nout)):
        r[name + "_comp"], r[name + "_index"], r[name + "_outer"] = take("<i4", n), take("<i4", n), take("<i4", n)
        r[name + "_area"], r[name + "_sign"] = take("<f8", n), take("<f8", n)
    r["u"] = take("<f8", (Nx + 1) * Ny * Nz)
    r["v"] = take("<f8", Nx * (Ny + 1) * Nz)
    r["w"] = take("<f8", Nx * Ny * (Nz + 1)) if dim == 3 else np.zeros(0)
    r["p"] = take("<f8", Nx * Ny * Nz)
    assert off == len(data), "trailing bytes in the result"
    return r


def run_bc(case, u, v, w, p, time=0.0, timeout=600) -> dict:
    """The reference's EnforceVelocityBC + EnforcePressureBC on the given fields (labels from the scene text)."""
    if not available():
        raise RuntimeError("oracle/_ref/ref_harness is not built (make -C oracle ref)")
    with tempfile.TemporaryDirectory() as td:
        cp, rp = os.path.join(td, "case.bin"), os.path.join(td, "res.bin")
        write_case(cp, case, u, v, w, scheme=SCHEME_BC_REPLAY, p_prev=p, time=time)
        r = subprocess.run([HARNESS, cp, rp], capture_output=True, text=True, timeout=timeout, cwd=td)
        if r.returncode != 0:
            raise RuntimeError("ref_harness failed (%d): %s %s" % (r.returncode, r.stdout[-2000:], r.stderr[-2000:]))
        return read_bc_result(rp, case.grid.dim)
