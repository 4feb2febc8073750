"""Synthetic pressure-projection cases: grids, spacing tables, scenes and seeded face velocities.

Every case the tests and the benchmark run is built here, once, on the host; the B200 path and the oracle then read
the same arrays, so no random-number library enters a comparison.

Conventions follow the NEREUS MAC grid (src/headers/Core/MAC.h:235-254, 369-374):
  * cell (i, j, k) = (y, x, z) at ``(i*Nx + j)*Nz + k``; ``Nx, Ny, Nz`` include the one-cell border ring;
  * ``u`` has ``Nx+1`` entries along x, ``v`` ``Ny+1`` along y, ``w`` ``Nz+1`` along z;
  * a 2D grid is the same layout with ``Nz = 1`` and no ``w``.
Spacing tables are the reference's padded ones (MAC.h:439-448): ``width[a][n+1] = Width(a, n)`` for n = -1..N and
``gap[a][n+1] = FaceGap(a, n)`` for n = -1..N-1, built as src/MAC.cpp:43-175 and 519-525 build them.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence

import numpy as np

# Cell types (src/headers/Core/Definitions.h:191-196).
FLUID, SOLID, EMPTY, INFLOW, PRESSURE, OUTFLOW = 0, 1, 2, 3, 4, 5
# Boundary kinds (Definitions.h:212).
BC_NOSLIP, BC_SLIP, BC_MOVING, BC_INLET, BC_PRESSURE_OUTLET, BC_OUTFLOW = 0, 1, 2, 3, 4, 5
FACE_NAMES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")
BC_NAMES = {BC_NOSLIP: "noslip", BC_SLIP: "slip", BC_MOVING: "moving", BC_INLET: "inflow",
            BC_PRESSURE_OUTLET: "pressure_outlet", BC_OUTFLOW: "outflow"}
PRIM_BOX, PRIM_SPHERE, PRIM_CYLINDER, PRIM_PLANE = 0, 1, 2, 3
REGION_SOLID, REGION_FLUID, REGION_EMPTY = 0, 1, 2


# --------------------------------------------------------------------------------------------------------------------
# spacing tables
# --------------------------------------------------------------------------------------------------------------------
@dataclasses.dataclass
class Axis:
    """One axis, ring included: cell widths, face and centre coordinates (N, N+1, N entries)."""

    size: np.ndarray
    face: np.ndarray
    centre: np.ndarray

    @property
    def n(self) -> int:
        return int(self.size.shape[0])

    def width_table(self) -> np.ndarray:
        """PadTable (MAC.h:519-525): entry n at [n+1], the edge value repeated at both ends."""
        s = self.size
        return np.concatenate([s[:1], s, s[-1:]]).astype(np.float64)

    def gap_table(self) -> np.ndarray:
        """GapTable (src/MAC.cpp:165-175): 0.5*(w[m] + w[m+1]) for m = -1..N-1, indices clamped."""
        w = self.size
        n = w.shape[0]
        a = w[np.clip(np.arange(-1, n), 0, n - 1)]
        b = w[np.minimum(np.arange(0, n + 1), n - 1)]
        return 0.5 * (a + b)


def _add_ring(size: List[float], face: List[float], centre: List[float]) -> Axis:
    """MAC::AddRing (src/MAC.cpp:150-161): one mirrored cell outside each end."""
    w0, w1 = size[0], size[-1]
    a0, a1 = face[0], face[-1]
    size = [w0] + list(size) + [w1]
    face = [a0 - w0] + list(face) + [a1 + w1]
    centre = [a0 - 0.5 * w0] + list(centre) + [a1 + 0.5 * w1]
    return Axis(np.array(size, dtype=np.float64), np.array(face, dtype=np.float64),
                np.array(centre, dtype=np.float64))


def uniform_axis(a0: float, n: int, dh: float) -> Axis:
    """MAC::BuildAxis's uniform branch (src/MAC.cpp:60-71) plus the ring: faces a0 + j*dh, centres a0 + j*dh + dh/2."""
    size = [dh] * n
    face = [a0 + j * dh for j in range(n + 1)]
    centre = [(a0 + j * dh) + dh / 2.0 for j in range(n)]
    return _add_ring(size, face, centre)


def explicit_axis(a0: float, widths: Sequence[float]) -> Axis:
    """A graded axis from its interior widths, laid out as MAC::BuildAxis lays out a graded span
    (src/MAC.cpp:137-145): running-sum faces, the last face pinned, centres halfway."""
    widths = [float(x) for x in widths]
    n = len(widths)
    face = [a0]
    for j in range(n):
        face.append(face[j] + widths[j])
    a_end = a0
    for x in widths:
        a_end += x
    face[n] = a_end
    centre = [0.5 * (face[j] + face[j + 1]) for j in range(n)]
    return _add_ring(widths, face, centre)


def band_stretched_widths(n_total: int, length: float, band_cells: int, band_centre: float,
                          growth: float) -> np.ndarray:
    """Interior widths of an axis with a uniform band of ``band_cells`` cells centred at ``band_centre`` and cell
    widths growing geometrically by ``growth`` per cell away from it on both sides.

    The band width h0 and the integer split nL + nR = n_total - band_cells are chosen so that each geometric side
    sums as closely as possible to its length (band_centre - band/2 and length - band_centre - band/2); each side is
    then rescaled to land exactly, the way MAC::BuildAxis rescales a graded span (src/MAC.cpp:130-133)."""
    half = band_cells // 2
    n_sides = n_total - band_cells
    left_len_of = lambda h0: band_centre - half * h0
    right_len_of = lambda h0: (length - band_centre) - half * h0

    def geo_sum(m: int) -> float:
        return sum(growth ** q for q in range(1, m + 1))

    best = None
    for n_left in range(1, n_sides):
        n_right = n_sides - n_left
        h_l = band_centre / (half + geo_sum(n_left))
        h_r = (length - band_centre) / (half + geo_sum(n_right))
        mismatch = abs(h_l - h_r) / h_l
        if best is None or mismatch < best[0]:
            best = (mismatch, n_left, n_right, 0.5 * (h_l + h_r))
    _, n_left, n_right, h0 = best
    left = np.array([h0 * growth ** q for q in range(n_left, 0, -1)])
    right = np.array([h0 * growth ** q for q in range(1, n_right + 1)])
    left *= left_len_of(h0) / left.sum()
    right *= right_len_of(h0) / right.sum()
    band = np.full(band_cells, h0)
    return np.concatenate([left, band, right])


@dataclasses.dataclass
class Grid:
    """A MAC grid's geometry: sizes (ring included), uniform dh, and the three axes."""

    dim: int
    axes: List[Axis]  # x, y, z
    dh: float
    nonuniform: bool
    domain: tuple  # (x0, xf, y0, yf, z0, zf)
    grid_size: int = 0  # GRID_SIZE for a uniform grid (MAC::InitializeGrid), 0 for explicit widths
    interior_widths: Optional[List[np.ndarray]] = None

    @property
    def Nx(self) -> int:
        return self.axes[0].n

    @property
    def Ny(self) -> int:
        return self.axes[1].n

    @property
    def Nz(self) -> int:
        return self.axes[2].n if self.dim == 3 else 1

    @property
    def shape(self):
        return (self.Ny, self.Nx, self.Nz)

    @property
    def cells(self) -> int:
        return self.Nx * self.Ny * self.Nz

    def u_shape(self):
        return (self.Ny, self.Nx + 1, self.Nz)

    def v_shape(self):
        return (self.Ny + 1, self.Nx, self.Nz)

    def w_shape(self):
        return (self.Ny, self.Nx, self.Nz + 1) if self.dim == 3 else (0,)

    def width_tables(self):
        return [self.axes[a].width_table() for a in range(3)]

    def gap_tables(self):
        return [self.axes[a].gap_table() for a in range(3)]

    def sample_coords(self, at_centre: bool):
        """The coordinate Scene::AxisCoord samples each cell at (Scene.h:623-634): its centre, or its low face."""
        return [ax.centre.copy() if at_centre else ax.face[: ax.n].copy() for ax in self.axes]


def uniform_grid(dim: int, domain: tuple, grid_size: int) -> Grid:
    """MAC::InitializeGrid (src/MAC.cpp:275-300, 2D :375-404): GRID_SIZE cells across the shortest side."""
    lx, ly = domain[1] - domain[0], domain[3] - domain[2]
    # InitializeGrid compares x and y only: z never sets dh.
    mn = ly if ly < lx else lx
    dh = mn / float(grid_size)
    cells = lambda L: int(L / dh + 1e-9)
    ax = uniform_axis(domain[0], cells(lx), dh)
    ay = uniform_axis(domain[2], cells(ly), dh)
    if dim == 3:
        az = uniform_axis(domain[4], cells(domain[5] - domain[4]), dh)
    else:
        az = Axis(np.array([dh]), np.array([0.0, dh]), np.array([dh / 2.0]))
    return Grid(dim, [ax, ay, az], dh, False, tuple(domain), grid_size=grid_size)


def stretched_grid(dim: int, domain: tuple, widths: Sequence[np.ndarray]) -> Grid:
    """A rectilinear grid from explicit interior widths per axis (the reference's stretched tables)."""
    ax = explicit_axis(domain[0], widths[0])
    ay = explicit_axis(domain[2], widths[1])
    if dim == 3:
        az = explicit_axis(domain[4], widths[2])
    else:
        w0 = float(widths[0][0])
        az = Axis(np.array([w0]), np.array([0.0, w0]), np.array([w0 / 2.0]))
    hmin = min(float(np.min(w)) for w in widths[:dim])
    hmin = min(hmin, float(ax.size.min()), float(ay.size.min()))
    return Grid(dim, [ax, ay, az], hmin, True, tuple(domain), grid_size=0,
                interior_widths=[np.asarray(w, dtype=np.float64) for w in widths[:dim]])


# --------------------------------------------------------------------------------------------------------------------
# scenes
# --------------------------------------------------------------------------------------------------------------------
@dataclasses.dataclass
class Region:
    region: int  # REGION_SOLID / FLUID / EMPTY
    kind: int  # PRIM_*
    p0: tuple = (0.0, 0.0, 0.0)
    p1: tuple = (0.0, 0.0, 0.0)
    radius: float = 0.0
    axis: int = 2
    invert: bool = False


@dataclasses.dataclass
class Scene:
    """The part of a NEREUS scene the pressure path sees: the six faces' kinds (in declaration order) and the
    interior regions, sampled at cell centres or corners (src/headers/Core/Scene.h:639-686)."""

    faces: List[tuple]  # (face index 0..5, BoundaryKind, has_p) in declaration order
    regions: List[Region]
    at_centre: bool = True
    pressure_expr: Optional[str] = None  # the p="..." of pressure-outlet faces with has_p
    face_params: Optional[dict] = None  # face index -> extra boundary parameters (u="..." v="..." w="...")
    pressure_exprs: Optional[dict] = None  # face index -> its own p="..." (else pressure_expr)

    def face_arrays(self):
        kind = [BC_NOSLIP] * 6
        has_p = [0] * 6
        order = [-1] * 6
        for n, (f, k, hp) in enumerate(self.faces):
            kind[f], has_p[f], order[f] = k, int(hp), n
        return kind, has_p, order

    def to_text(self) -> str:
        """The scene file the reference's Scene::LoadText reads for the same geometry."""
        g = lambda x: "%.17g" % x
        lines = ["sampling %s" % ("center" if self.at_centre else "corner")]
        for f, k, hp in self.faces:
            line = "boundary %s %s" % (FACE_NAMES[f], BC_NAMES[k])
            if hp:
                expr = (self.pressure_exprs or {}).get(f, self.pressure_expr or "0")
                line += ' p="%s"' % expr
            if self.face_params and f in self.face_params:
                line += " " + self.face_params[f]
            lines.append(line)
        for r in self.regions:
            kind = {REGION_SOLID: "solid", REGION_FLUID: "fluid", REGION_EMPTY: "empty"}[r.region]
            prim = {PRIM_BOX: "box", PRIM_SPHERE: "sphere", PRIM_CYLINDER: "cylinder", PRIM_PLANE: "plane"}[r.kind]
            t = lambda v: "(%s,%s,%s)" % (g(v[0]), g(v[1]), g(v[2]))
            parts = ["region", kind, prim]
            if r.kind == PRIM_BOX:
                parts += ["min=" + t(r.p0), "max=" + t(r.p1)]
            elif r.kind == PRIM_PLANE:
                parts += ["point=" + t(r.p0), "normal=" + t(r.p1)]
            else:
                parts += ["center=" + t(r.p0), "radius=" + g(r.radius)]
                if r.kind == PRIM_CYLINDER:
                    parts.append("axis=" + "xyz"[r.axis])
            if r.invert:
                parts.append("invert=1")
            lines.append(" ".join(parts))
        return "\n".join(lines) + "\n"


def walls_scene(dim: int, outlet_face: Optional[int] = None, inlet_face: Optional[int] = None,
                regions: Sequence[Region] = (), at_centre: bool = True) -> Scene:
    """No-slip walls on every face, with an optional p = 0 pressure outlet and velocity inlet. The walls are
    declared first, the inlet and outlet last, so those win the ring's edges."""
    nf = 6 if dim == 3 else 4
    faces = [(f, BC_NOSLIP, 0) for f in range(nf) if f not in (outlet_face, inlet_face)]
    if inlet_face is not None:
        faces.append((inlet_face, BC_INLET, 0))
    if outlet_face is not None:
        faces.append((outlet_face, BC_PRESSURE_OUTLET, 0))
    return Scene(faces, list(regions), at_centre)


# --------------------------------------------------------------------------------------------------------------------
# seeded normal face velocities: SplitMix64 (counter based) -> Box-Muller
# --------------------------------------------------------------------------------------------------------------------
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, start: int, count: int) -> np.ndarray:
    """The SplitMix64 outputs number start..start+count-1 of the stream keyed by ``seed``."""
    with np.errstate(over="ignore"):
        idx = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + idx * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def normals(seed: int, count: int) -> np.ndarray:
    """``count`` N(0,1) draws: pairs of (0,1] uniforms from SplitMix64, Box-Muller."""
    pairs = (count + 1) // 2
    z = splitmix64(seed, 0, 2 * pairs)
    u = ((z >> np.uint64(11)).astype(np.float64) + 1.0) * (1.0 / 9007199254740992.0)
    u1, u2 = u[0::2], u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    t = 2.0 * math.pi * u2
    out = np.empty(2 * pairs)
    out[0::2] = r * np.cos(t)
    out[1::2] = r * np.sin(t)
    return out[:count]


def stream_seed(seed: int, stream: int) -> int:
    return int(splitmix64(seed, stream, 1)[0])


def face_velocities(grid: Grid, types: np.ndarray, seed: int, rule: str = "solid", fp32: bool = False):
    """N(0,1) face velocities u, v (, w), one stream per component.

    ``rule='solid'``: every face with a SOLID cell on either side, or outside the grid, is zeroed
    (MAC::BuildSolidFaceList3D/2D + EnforceVelocityBC, src/MAC.cpp:837-845, 1010-1041).
    ``rule='liquid'``: only faces with a FLUID side and no SOLID side keep their draw (free-surface tanks).
    ``rule='zero'``: every face 0 (the known-answer cases).
    ``fp32``: the draws are rounded to float32 first (then held as float64)."""
    t = types.reshape(grid.shape)
    if rule == "zero":
        z = [np.zeros(int(np.prod(s))).reshape(s) for s in (grid.u_shape(), grid.v_shape())]
        z.append(np.zeros(int(np.prod(grid.w_shape()))).reshape(grid.w_shape()) if grid.dim == 3 else np.zeros(0))
        return z
    out = []
    comps = 3 if grid.dim == 3 else 2
    for c in range(comps):
        shape = [grid.u_shape(), grid.v_shape(), grid.w_shape()][c]
        vals = normals(stream_seed(seed, c), int(np.prod(shape))).reshape(shape)
        if fp32:
            vals = vals.astype(np.float32).astype(np.float64)
        pad = [(0, 0)] * 3
        pad[[1, 0, 2][c]] = (1, 1)
        tp = np.pad(t, pad, constant_values=SOLID)
        ax = [1, 0, 2][c]
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax] = slice(0, -1)
        hi[ax] = slice(1, None)
        a, b = tp[tuple(lo)], tp[tuple(hi)]
        if rule == "solid":
            keep = (a != SOLID) & (b != SOLID)
        else:
            keep = (a != SOLID) & (b != SOLID) & ((a == FLUID) | (b == FLUID))
        vals = np.where(keep, vals, 0.0)
        out.append(np.ascontiguousarray(vals, dtype=np.float64))
    if comps == 2:
        out.append(np.zeros(0, dtype=np.float64))
    return out


# --------------------------------------------------------------------------------------------------------------------
# the named cases
# --------------------------------------------------------------------------------------------------------------------
@dataclasses.dataclass
class Case:
    name: str
    grid: Grid
    scene: Scene
    seed: int
    rho: float = 1.0
    dt: float = 1e-3
    needs_compat: bool = False
    tol: float = 1e-8
    velocity_rule: str = "solid"
    fp32_velocity: bool = False
    method: int = 0  # 0 Eulerian (ADI-like, fixed region), 1 hybrid (FLIP-like)


def closed_box_2d(n: int = 128, seed: int = 1) -> Case:
    """2D closed box, uniform n x n on the unit square, all interior fluid, no-slip walls: all-Neumann (singular,
    compatibility condition on)."""
    g = uniform_grid(2, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    return Case("closed_box_2d_%d" % n, g, walls_scene(2), seed, needs_compat=True, tol=1e-10)


def sphere_outlet_3d(n: int = 256, seed: int = 2) -> Case:
    """3D unit cube, uniform n^3, a solid sphere at (0.5, 0.5, 0.5) radius 0.15 sampled at cell centres, no-slip walls
    and a p = 0 pressure outlet on the x = 1 face."""
    g = uniform_grid(3, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    sph = Region(REGION_SOLID, PRIM_SPHERE, (0.5, 0.5, 0.5), radius=0.15)
    return Case("sphere_outlet_3d_%d" % n, g, walls_scene(3, outlet_face=1, regions=[sph]), seed)


def stretched_cylinder_3d(nx: int = 192, ny: int = 128, nz: int = 128, seed: int = 3) -> Case:
    """3D channel [0,2.2]x[0,0.41]^2, x stretched by 1.04 away from a 24-cell band centred at x = 0.5 (scaled with
    nx), a solid cylinder along z at (0.5, 0.2) radius 0.05, a velocity inlet at x = 0 (Neumann), a p = 0 outlet at
    x = 2.2 and no-slip walls."""
    band = max(2, (24 * nx) // 192 // 2 * 2)
    wx = band_stretched_widths(nx, 2.2, band, 0.5, 1.04)
    wy = np.full(ny, 0.41 / ny)
    wz = np.full(nz, 0.41 / nz)
    g = stretched_grid(3, (0.0, 2.2, 0.0, 0.41, 0.0, 0.41), [wx, wy, wz])
    cyl = Region(REGION_SOLID, PRIM_CYLINDER, (0.5, 0.2, 0.0), radius=0.05, axis=2)
    return Case("stretched_cylinder_3d_%dx%dx%d" % (nx, ny, nz), g,
                walls_scene(3, outlet_face=1, inlet_face=0, regions=[cyl]), seed)


def flip_tank_3d(n: int = 128, seed: int = 4, a: Optional[float] = None, b: Optional[float] = None) -> Case:
    """A FLIP-style free-surface tank: unit cube, uniform n^3, interior cells with centre x < a and z < b liquid
    (FLUID), the other interior cells air (EMPTY, p = 0), solid walls. a, b ~ U(0.3, 0.7) from the seed unless
    given. Liquid-face velocities are N(0,1) rounded to FP32."""
    if a is None or b is None:
        z = splitmix64(seed, 1000, 2)
        uu = ((z >> np.uint64(11)).astype(np.float64) + 1.0) * (1.0 / 9007199254740992.0)
        a = 0.3 + 0.4 * float(uu[0]) if a is None else a
        b = 0.3 + 0.4 * float(uu[1]) if b is None else b
    g = uniform_grid(3, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    air = Region(REGION_EMPTY, PRIM_BOX, (-1.0, -1.0, -1.0), (2.0, 2.0, 2.0))
    liquid = Region(REGION_FLUID, PRIM_BOX, (-1.0, -1.0, -1.0), (a, 2.0, b))
    sc = walls_scene(3, regions=[air, liquid])
    return Case("flip_tank_3d_%d_a%.4f_b%.4f" % (n, a, b), g, sc, seed, velocity_rule="liquid",
                fp32_velocity=True, method=1)


def bc_channel_3d(n: int = 12, seed: int = 23) -> Case:
    """Every boundary kind the velocity replay handles, on a unit cube n^3 with a solid sphere at (0.5, 0.5, 0.5)
    radius 0.2: a space- and time-dependent inlet at x = 0, an outflow (continuity) at x = 1, slip walls at y = 0
    and y = 1, a wall sliding along x at z = 1 and a no-slip wall at z = 0."""
    g = uniform_grid(3, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    sphere = Region(REGION_SOLID, PRIM_SPHERE, (0.5, 0.5, 0.5), radius=0.2)
    faces = [(4, BC_NOSLIP, 0), (2, BC_SLIP, 0), (3, BC_SLIP, 0), (5, BC_MOVING, 0), (0, BC_INLET, 0),
             (1, BC_OUTFLOW, 0)]
    params = {0: 'u="1+0.25*sin(3*t)*y" v="0.1*z" w="0"', 5: 'u="0.5+t"'}
    return Case("bc_channel_3d_%d" % n, g, Scene(faces, [sphere], True, None, params), seed)


def bc_outlet_2d(n: int = 20, seed: int = 24) -> Case:
    """The 2D replay with a prescribed outlet pressure: unit square n^2, a parabolic inlet at x = 0, a pressure
    outlet p = 0.1 t + y at x = 1, a slip wall at y = 0, a no-slip wall at y = 1."""
    g = uniform_grid(2, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    faces = [(3, BC_NOSLIP, 0), (2, BC_SLIP, 0), (0, BC_INLET, 0), (1, BC_PRESSURE_OUTLET, 1)]
    params = {0: 'u="4*y*(1-y)" v="0"'}
    return Case("bc_outlet_2d_%d" % n, g, Scene(faces, [], True, "0.1*t+y", params), seed)


def bc_suite_scene(scene: int, dim: int, seed: int = 29, stretched: bool = False) -> Case:
    """The four scenes of the reference's own boundary-condition test (tests/suite_units.cpp:453-480), on its grids
    (unit square 24^2 or unit cube 12^3, uniform):
    0 a closed box with a moving lid (u = 1, w = 0.5 x), a slip side, walls and an interior solid box;
    1 a channel with a time-dependent inlet and pressure outlets on three faces meeting at corners, a solid sphere;
    2 prescribed pressures on three faces, an outlet at p = 0, an inlet, a slip wall, a solid box;
    3 an inlet whose flux leaves through a continuity outflow, slip walls, a solid sphere.
    ``stretched`` grades y and z by 1.15 per cell away from a 4-cell band (the reference's test grades its grids too).
    """
    n = 24 if dim == 2 else 12
    if stretched:
        # graded in y and z (x uniform), so the faces of an x boundary differ in area
        wy = band_stretched_widths(n, 1.0, 4, 0.75, 1.15)
        wz = band_stretched_widths(n, 1.0, 4, 0.15, 1.15)
        g = stretched_grid(dim, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), [np.full(n, 1.0 / n), wy, wz][:dim])
    else:
        g = uniform_grid(dim, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    XMIN, XMAX, YMIN, YMAX, ZMIN, ZMAX = range(6)
    if scene == 0:
        faces = [(XMIN, BC_NOSLIP, 0), (XMAX, BC_SLIP, 0), (YMIN, BC_NOSLIP, 0), (ZMIN, BC_SLIP, 0),
                 (ZMAX, BC_NOSLIP, 0), (YMAX, BC_MOVING, 0)]
        params, pexprs = {YMAX: 'u="1" w="0.5*x"'}, None
        regions = [Region(REGION_SOLID, PRIM_BOX, (0.35, 0.3, 0.3), (0.6, 0.55, 0.6))]
    elif scene == 1:
        faces = [(XMIN, BC_INLET, 0), (XMAX, BC_PRESSURE_OUTLET, 0), (YMIN, BC_NOSLIP, 0),
                 (ZMIN, BC_PRESSURE_OUTLET, 0), (ZMAX, BC_NOSLIP, 0), (YMAX, BC_PRESSURE_OUTLET, 0)]
        params, pexprs = {XMIN: 'u="1 + 0.5*sin(3*t) + y" v="0.2*y" w="0.1*z"'}, None
        regions = [Region(REGION_SOLID, PRIM_SPHERE, (0.5, 0.5, 0.5), radius=0.18)]
    elif scene == 2:
        faces = [(XMIN, BC_PRESSURE_OUTLET, 1), (XMAX, BC_PRESSURE_OUTLET, 1), (YMIN, BC_PRESSURE_OUTLET, 0),
                 (YMAX, BC_INLET, 0), (ZMIN, BC_PRESSURE_OUTLET, 1), (ZMAX, BC_SLIP, 0)]
        params = {YMAX: 'u="0.2" v="-0.5*x" w="0"'}
        pexprs = {XMIN: "1 + y + t", XMAX: "0.5*t - x", ZMIN: "2*z"}
        regions = [Region(REGION_SOLID, PRIM_BOX, (0.4, 0.4, 0.4), (0.6, 0.7, 0.55))]
    else:
        faces = [(XMIN, BC_INLET, 0), (XMAX, BC_OUTFLOW, 0), (YMIN, BC_NOSLIP, 0), (YMAX, BC_SLIP, 0),
                 (ZMIN, BC_SLIP, 0), (ZMAX, BC_SLIP, 0)]
        params, pexprs = {XMIN: 'u="1 - (y - 1)^2 + 0.3*z"'}, None
        regions = [Region(REGION_SOLID, PRIM_SPHERE, (0.5, 0.4, 0.5), radius=0.15)]
    sc = Scene(faces, regions, True, None, params, pexprs)
    return Case("bc_suite_scene%d_%dd_%d%s" % (scene, dim, n, "_stretched" if stretched else ""), g, sc, seed)


def flip_tank_2d(n: int = 32, seed: int = 10, a: float = 0.55, b: float = 0.45) -> Case:
    """A 2D FLIP-style tank: unit square, uniform n^2, interior cells with centre x < a and y < b liquid (FLUID), the
    rest air (EMPTY), no-slip walls and an open top (a pressure outlet without p=, so its ring cells are EMPTY)."""
    g = uniform_grid(2, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    air = Region(REGION_EMPTY, PRIM_BOX, (-1.0, -1.0, -1.0), (2.0, 2.0, 2.0))
    liquid = Region(REGION_FLUID, PRIM_BOX, (-1.0, -1.0, -1.0), (a, b, 2.0))
    return Case("flip_tank_2d_%d" % n, g, walls_scene(2, outlet_face=3, regions=[air, liquid]), seed,
                velocity_rule="liquid", fp32_velocity=True, method=1)


def _uniforms(seed: int, stream: int, count: int) -> np.ndarray:
    z = splitmix64(stream_seed(seed, stream), 0, count)
    return ((z >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)


def flip_particles(case: Case, types: np.ndarray, seed: int, ppc: int = 4, hole_fraction: float = 0.03,
                   features: bool = True) -> np.ndarray:
    """Seeded FLIP particle positions, (count, 3) float64 (z = 0 in 2D), for a relabelling step on ``case``:
    ``ppc`` particles jittered uniformly inside every interior FLUID cell of ``types``, except that the cells of
    a ``hole_fraction`` draw hold none. With ``features``, also: straight runs of 4 empty cells along each axis
    inside the liquid (each filled only when its lower neighbour was filled first); a 2 x 2 block of empty cells; a
    few spray particles in air; particles exactly on a face coordinate, within one cell below the grid's first face,
    and far beyond its last face (the index clamp)."""
    g = case.grid
    t = types.reshape(g.shape)
    nd = g.dim
    faces = [ax.face for ax in g.axes]  # x, y, z face coordinates, ring included
    dh = g.dh
    liquid = np.zeros(g.shape, dtype=bool)
    sl = tuple(slice(1, -1) for _ in range(nd)) + (() if nd == 3 else (slice(None),))
    liquid[sl] = t[sl] == FLUID
    cells = np.argwhere(liquid)  # (i, j, k) in the (y, x, z) layout
    drop = _uniforms(seed, 1, len(cells)) < hole_fraction
    if features and len(cells):
        lo, hi = cells.min(axis=0), cells.max(axis=0)
        mid = (lo + hi) // 2
        holes = set()
        axes = (0, 1, 2) if nd == 3 else (0, 1)
        for n_ax, ax in enumerate(axes):
            c0 = mid.copy()
            for other in axes:
                if other != ax:
                    c0[other] = min(max(lo[other] + 1, mid[other] + (2 * n_ax - 2)), hi[other] - 1)
            c0[ax] = max(lo[ax] + 1, mid[ax] - 2)
            for s in range(4):
                c = c0.copy()
                c[ax] = min(c0[ax] + s, hi[ax] - 1)
                holes.add(tuple(int(v) for v in c))
        b0 = [min(max(lo[a] + 1, lo[a] + 1), hi[a] - 2) for a in range(3)]
        for di in (0, 1):
            for dj in (0, 1):
                holes.add((b0[0] + di, b0[1] + dj, b0[2]))
        for n_c, c in enumerate(cells):
            if tuple(int(v) for v in c) in holes:
                drop[n_c] = True
    keep = cells[~drop]
    r = _uniforms(seed, 2, len(keep) * ppc * 3).reshape(len(keep), ppc, 3)
    # (i, j, k) -> x from column j, y from row i, z from k
    x = faces[0][keep[:, 1]][:, None] + dh * r[:, :, 0]
    y = faces[1][keep[:, 0]][:, None] + dh * r[:, :, 1]
    z = faces[2][keep[:, 2]][:, None] + dh * r[:, :, 2] if nd == 3 else np.zeros_like(x)
    pts = [np.stack([x.reshape(-1), y.reshape(-1), z.reshape(-1)], axis=1)]
    if features:
        ext = []
        air = np.argwhere(t == EMPTY)
        if len(air):
            pick = (_uniforms(seed, 3, 3) * len(air)).astype(np.int64)
            for q in pick:
                i, j, k = air[q]
                ext.append([faces[0][j] + 0.5 * dh, faces[1][i] + 0.5 * dh,
                            faces[2][k] + 0.5 * dh if nd == 3 else 0.0])
        zc = faces[2][g.Nz // 2] + 0.25 * dh if nd == 3 else 0.0
        ext.append([faces[0][2], faces[1][2], faces[2][2] if nd == 3 else 0.0])  # exactly on faces
        ext.append([faces[0][0] - 0.4 * dh, faces[1][1] + 0.5 * dh, zc])  # within one cell below the first face
        ext.append([faces[0][g.Nx // 2] + 0.5 * dh, faces[1][-1] + 7.0 * dh, zc])  # beyond the top: clamped
        ext.append([1.0e3, faces[1][g.Ny // 2], zc])  # far beyond x: clamped
        pts.append(np.array(ext, dtype=np.float64))
    return np.ascontiguousarray(np.concatenate(pts, axis=0))


def channel_2d_stretched(nx: int = 24, ny: int = 12, seed: int = 5) -> Case:
    """2D channel [0,2.2]x[0,0.41], x stretched by 1.04 away from a band at x = 0.5, a solid disc at (0.5, 0.2)
    radius 0.05, inlet at x = 0, p = 0 outlet at x = 2.2."""
    band = max(2, (nx // 8) // 2 * 2)
    wx = band_stretched_widths(nx, 2.2, band, 0.5, 1.04)
    wy = np.full(ny, 0.41 / ny)
    g = stretched_grid(2, (0.0, 2.2, 0.0, 0.41, 0.0, 1.0), [wx, wy])
    disc = Region(REGION_SOLID, PRIM_CYLINDER, (0.5, 0.2, 0.0), radius=0.05, axis=2)
    return Case("channel_2d_stretched_%dx%d" % (nx, ny), g, walls_scene(2, outlet_face=1, inlet_face=0,
                                                                         regions=[disc]), seed)


def cavity_outlet_2d(n: int = 32, seed: int = 9) -> Case:
    """2D unit square, uniform n x n, a solid disc at (0.4, 0.5) radius 0.15, no-slip walls and a p = 0 pressure outlet
    on the x = 1 face: a uniform 2D scene of the kind the EXPLICIT method runs."""
    g = uniform_grid(2, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    disc = Region(REGION_SOLID, PRIM_CYLINDER, (0.4, 0.5, 0.0), radius=0.15, axis=2)
    return Case("cavity_outlet_2d_%d" % n, g, walls_scene(2, outlet_face=1, regions=[disc]), seed)


def inflow_outflow_3d(n: int = 8, seed: int = 6) -> Case:
    """3D unit cube with a velocity inlet at x = 0 and a continuity outflow at x = 1 (both Neumann for the
    pressure: a singular system, compatibility on)."""
    g = uniform_grid(3, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    faces = [(f, BC_NOSLIP, 0) for f in (2, 3, 4, 5)] + [(0, BC_INLET, 0), (1, BC_OUTFLOW, 0)]
    return Case("inflow_outflow_3d_%d" % n, g, Scene(faces, [], True), seed, needs_compat=True)


def all_solid_3d(n: int = 6, seed: int = 7) -> Case:
    """Every interior cell solid: no unknowns at all."""
    g = uniform_grid(3, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    box = Region(REGION_SOLID, PRIM_BOX, (-1.0, -1.0, -1.0), (2.0, 2.0, 2.0))
    return Case("all_solid_3d_%d" % n, g, walls_scene(3, regions=[box]), seed)


def dirichlet_linear_2d(n: int = 40) -> Case:
    """The reference's known-answer case (tests/suite_pressure.cpp:55-57, 68-76, 84-97): every face a pressure
    outlet prescribing p = 0.3 + 1.1x - 0.7y, corner sampling, zero velocity; the linear field is exact."""
    g = uniform_grid(2, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    faces = [(f, BC_PRESSURE_OUTLET, 1) for f in range(4)]
    return Case("dirichlet_linear_2d_%d" % n, g, Scene(faces, [], False, "0.3 + 1.1*x - 0.7*y"), 0, tol=1e-9,
                velocity_rule="zero")


def dirichlet_linear_3d(n: int = 20) -> Case:
    g = uniform_grid(3, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    faces = [(f, BC_PRESSURE_OUTLET, 1) for f in range(6)]
    return Case("dirichlet_linear_3d_%d" % n, g, Scene(faces, [], False, "0.3 + 1.1*x - 0.7*y"), 0, tol=1e-12,
                velocity_rule="zero")


def pressure_outlet_3d(n: int = 12, seed: int = 8) -> Case:
    """3D unit cube, uniform n^3, a solid sphere at (0.5, 0.5, 0.5) radius 0.2, no-slip walls and a pressure outlet
    on x = 1 that prescribes a time-dependent p = 0.2 + 0.5 t + 0.3 y (PRESSURE ring cells: the incremental
    scheme's Dirichlet increments p_b(t^{n+1}) - p_b(t^n) are non-zero)."""
    g = uniform_grid(3, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), n)
    sph = Region(REGION_SOLID, PRIM_SPHERE, (0.5, 0.5, 0.5), radius=0.2)
    faces = [(f, BC_NOSLIP, 0) for f in (0, 2, 3, 4, 5)] + [(1, BC_PRESSURE_OUTLET, 1)]
    return Case("pressure_outlet_3d_%d" % n, g, Scene(faces, [sph], True, PRESSURE_OUTLET_EXPR), seed)


PRESSURE_OUTLET_EXPR = "0.2 + 0.5*t + 0.3*y"


def outlet_pressure(t):
    """p_b of pressure_outlet_3d at time t, as a function of the ring face position."""
    return lambda x, y, z=0.0: 0.2 + 0.5 * t + 0.3 * y


def previous_pressure(grid: Grid, types: np.ndarray, seed: int, ring_fn=None) -> np.ndarray:
    """A previous step's pressure p^n for the incremental scheme and the warm start: seeded N(0,1) values on the
    interior FLUID cells (stream 7 of the case seed), the prescribed values ring_fn(x, y, z) on PRESSURE ring cells,
    0 elsewhere."""
    t = np.asarray(types).reshape(-1)
    p = ring_prescribed_pressure(grid, t, ring_fn) if ring_fn is not None else np.zeros(grid.cells)
    tv = t.reshape(grid.shape)
    interior = np.zeros(grid.shape, dtype=bool)
    if grid.dim == 3:
        interior[1:-1, 1:-1, 1:-1] = True
    else:
        interior[1:-1, 1:-1, :] = True
    fluid = (tv == FLUID) & interior
    vals = normals(stream_seed(seed, 7), int(fluid.sum()))
    pv = p.reshape(grid.shape)
    pv[fluid] = vals
    return p


def linear_pressure(x, y, z=0.0):
    """p_b of the known-answer case, evaluated where MAC::PrescribedPressure evaluates it."""
    return 0.3 + 1.1 * x - 0.7 * y


def ring_prescribed_pressure(grid: Grid, types: np.ndarray, fn) -> np.ndarray:
    """A pressure field holding, on every PRESSURE ring cell, fn at the boundary face the cell borders
    (MAC::PrescribedPressure, src/MAC.cpp:595-612), 0 elsewhere."""
    p = np.zeros(grid.cells)
    t = types.reshape(grid.shape)
    Nx, Ny, Nz = grid.Nx, grid.Ny, grid.Nz

    def ring_coord(a, n, N):
        ax = grid.axes[a]
        if n == 0:
            return ax.face[1]
        if n == N - 1:
            return ax.face[N - 1]
        return ax.centre[n]

    pv = p.reshape(grid.shape)
    for i, j, k in zip(*np.nonzero(t == PRESSURE)):
        x = ring_coord(0, j, Nx)
        y = ring_coord(1, i, Ny)
        z = ring_coord(2, k, Nz) if grid.dim == 3 else 0.0
        pv[i, j, k] = fn(x, y, z)
    return p
