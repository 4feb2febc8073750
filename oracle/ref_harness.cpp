// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into or called by the product library.
//
// A driver for the NEREUS reference's own pressure path, compiled from the reference sources where they lie
// (src/MAC.cpp, src/Utils.cpp, src/Methods/PPESolver/PressureSolver{2,3}D.cpp, src/Methods/Explicit/Explicit2D.cpp,
// src/Methods/FLIP/{FLIP,DiffusionSolver}{2,3}D.cpp, include/tinyexpr/tinyexpr.c) by
// oracle/Makefile into oracle/_ref/ref_harness. It reads one case file, drives the reference exactly the way its
// own harnesses do (tests/suite_pressure.cpp:84-122: build a MAC, set the cell types, InitializePressureSolver,
// SolvePressure, ProjectPressure), and writes what the reference computed:
//   cell types, IDP numbering, the assembled CSR matrix (PressureSolver3D::SYSTEM.A), the right-hand side b before
//   and after the compatibility step, the solution x, the pressure field after the solve, the projected face
//   velocities, iteration count, and wall times (steady_clock, as GetWallTime, src/Utils.cpp:50-53).
//
// Private members (the spacing tables, SYSTEM, DirichletSum) are reached by compiling THIS translation unit with
// `private` defined as `public`; the reference's own objects are compiled unchanged.
//
// Case file (little endian), written by oracle/refcase.py:
//   "NBCASE01", int32 hdr[16], double dom[6], double rho, dt, tol, time,
//   [grid_mode 1] double wx[nxi], wy[nyi], wz[nzi] (interior widths),
//   [label_mode 0] int32 len + scene text; [label_mode 1] uint8 labels[cells],
//   double u[], v[], (w[] in 3D), in the MAC layouts (MAC.h:235-242, 369-374),
//   [scheme 1 or 2] double p_prev[cells]: the previous step's pressure (gridAnt->p, ring included).
// hdr: dim, grid_mode, grid_size, nxi, nyi, nzi, label_mode, needs_compat, scheme, solver, max_iters, threads,
//      method_kind (0 Eulerian/ADI-like, 1 hybrid/FLIP-like), repeats, Nx, Ny (expected, ring included).
// scheme: 0 Chorin; 1 incremental (SolvePressure with SYSTEM.scheme = PRESSURE_INCREMENTAL from gridAnt, then
// ProjectPressure + AccumulatePressureIncrement as Project does); 2 Chorin with the warm start from gridAnt;
// 3 (2D, uniform) the EXPLICIT method's own pressure step and projection (src/Methods/Explicit/Explicit2D.cpp:48-120,
// SOR to tol * max|b| in the max norm with at most max_iters sweeps), after the shared assembly that A, IDP and b
// (written as for Chorin, with the relative residual of the SOR solution in that system) come from; iterations -1.
// 4 FLIP's re-labelling (FLIP3D::UpdateFluidCells, src/Methods/FLIP/FLIP3D.cpp:784-833; FLIP2D::UpdateFluidCells,
// src/Methods/FLIP/FLIP2D.cpp:648-691) from the particle positions of the case file, then the Chorin step on the new
// labels.
// With NB_REF_LEAN=1 in the environment the result leaves out cell types, IDP, the CSR matrix and both right-hand
// sides (nnz is written as 0 and the header's last double as 1.0), for grids where those run to gigabytes.
// [scheme 1 or 2] The result file then ends with double ref_norm (IncrementReferenceNorm, 0 for Chorin) and double
// p_final[cells] (the pressure after Project).
// [scheme 4] The case file ends with int64 count and double xyz[3 * count] (x, y, z per particle); the result file
// with double origin[3] (FacePos(X|Y|Z, 0)) and uint8 types_before[cells] (the labels UpdateFluidCells started from).
// 5 the boundary-condition replay alone (MAC::EnforceVelocityBC and EnforcePressureBC, src/MAC.cpp:613-871): the
// case file ends with double p[cells], the pressure the ring is enforced on; the boundary functions are the scene's.
// The result file is then "NBBC0001", int32 {Nx, Ny, Nz, nsolid[3], npresc, ncopy, nring, ninlet, noutflow}, the
// lists BuildBoundaryLists made, in their order (solidFaceList[c]; prescribedList as int32 c[], index[] and the
// double value the boundary function gave each entry at `time`; copyList as int32 c[], dst[], src[]; ringList as
// int32 dst[], kind[], src[] and double value[] (PrescribedPressure for kind 1, else 0); inletFaces then
// outflowFaces as int32 c[], index[], outer[], double area[], sign[]), then u, v, (w,) p after the two calls.
#include <algorithm>
#include <array>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <limits>
#include <map>
#include <memory>
#include <ostream>
#include <set>
#include <sstream>
#include <string>
#include <tuple>
#include <unordered_map>
#include <utility>
#include <vector>
#include <omp.h>
#include <Eigen/Dense>
#include <Eigen/Sparse>
#include <Eigen/IterativeLinearSolvers>
#define AMGCL_NO_BOOST
#include <amgcl/backend/builtin.hpp>
#include <amgcl/adapter/crs_tuple.hpp>
#include <amgcl/make_solver.hpp>
#include <amgcl/amg.hpp>
#include <amgcl/coarsening/smoothed_aggregation.hpp>
#include <amgcl/relaxation/spai0.hpp>
#include <amgcl/solver/cg.hpp>
#include <stl_reader/stl_reader.h>
#include <tmd/TriangleMeshDistance.h>
#include "tinyexpr.h"

// Only the reference's own class declarations below are opened up; every library header above is included first,
// untouched.
#define private public
#define protected public
#include "headers/Core/MAC.h"
#include "headers/Core/Definitions.h"
#include "headers/Core/Scene.h"
#include "Methods/PPESolver/PressureSolver2D.h"
#include "Methods/PPESolver/PressureSolver3D.h"
#include "Methods/Explicit/ExplicitSettings.h"
#include "Methods/FLIP/FLIP2D.h"
#include "Methods/FLIP/FLIP3D.h"
#undef private
#undef protected

static double Now()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class T> static void ReadN(FILE *f, T *dst, size_t n)
{
    if (n && std::fread(dst, sizeof(T), n, f) != n) { std::fprintf(stderr, "short read\n"); std::exit(3); }
}
template <class T> static void WriteN(FILE *f, const T *src, size_t n)
{
    if (n) std::fwrite(src, sizeof(T), n, f);
}

// A method row with the capabilities the pressure path asks about: Eulerian (fixed region, stretched grids allowed)
// or hybrid (FLIP-like: moving region, uniform only). Definitions.h:1096-1120.
static void RegisterHarnessMethod(int kind)
{
    METHOD_COUNT = 0;
    SimulationMethod m = {};
    m.key = kind == 0 ? "ORACLE_EULERIAN" : "ORACLE_HYBRID";
    m.label = m.key;
    m.help = "";
    m.family = kind == 0 ? MethodFamily::EULERIAN : MethodFamily::HYBRID;
    m.supports2D = m.supports3D = true;
    m.caps = kind == 0 ? (CAP_GRID | CAP_RECTILINEAR | CAP_BOUNDARY_CELLS | CAP_FIXED_REGION | CAP_PRESSURE_SOLVER)
                       : (CAP_GRID | CAP_BOUNDARY_CELLS | CAP_PRESSURE_SOLVER);
    SIM_TYPE = RegisterSimulationMethod(m);
}

// One stretched axis as MAC::BuildAxis lays out a graded span (src/MAC.cpp:137-145) plus MAC::AddRing
// (src/MAC.cpp:150-161), from the interior widths the case gives.
static void FillAxis(double a0, const std::vector<double> &wi, std::vector<double> &size, std::vector<double> &face,
                     std::vector<double> &centre)
{
    const int n = (int)wi.size();
    size = wi;
    face.assign(n + 1, 0.0);
    centre.assign(n, 0.0);
    face[0] = a0;
    for (int j = 0; j < n; j++) face[j + 1] = face[j] + size[j];
    double aEnd = a0;
    for (int j = 0; j < n; j++) aEnd += wi[j];
    face[n] = aEnd;
    for (int j = 0; j < n; j++) centre[j] = 0.5 * (face[j] + face[j + 1]);
    MAC::AddRing(size, face, centre);
}

// MAC::InitializeGrid + BuildSpacing (src/MAC.cpp:177-273, 275-317) for explicit interior widths.
static void InitStretched(MAC &g, int dim, const double *dom, const std::vector<double> &wx,
                          const std::vector<double> &wy, const std::vector<double> &wz)
{
    g.is2D = (dim == 2);
    g.omega = Domain{dom[0], dom[1], dom[2], dom[3], dom[4], dom[5]};
    g.nonUniform = true;
    FillAxis(dom[0], wx, g.dxs, g.xfv, g.xcv);
    FillAxis(dom[2], wy, g.dys, g.yfv, g.ycv);
    if (g.is2D)
    {
        g.dzs.assign(1, wx[0]);
        g.zfv.assign(2, 0.0);
        g.zfv[1] = wx[0];
        g.zcv.assign(1, wx[0] / 2.0);
    }
    else
        FillAxis(dom[4], wz, g.dzs, g.zfv, g.zcv);
    g.Nx = (int)g.dxs.size();
    g.Ny = (int)g.dys.size();
    g.Nz = g.is2D ? 0 : (int)g.dzs.size();
    MAC::PadTable(g.dxs, g.widthTable[MAC::X]); MAC::PadTable(g.dys, g.widthTable[MAC::Y]); MAC::PadTable(g.dzs, g.widthTable[MAC::Z]);
    MAC::PadTable(g.xfv, g.faceTable[MAC::X]);  MAC::PadTable(g.yfv, g.faceTable[MAC::Y]);  MAC::PadTable(g.zfv, g.faceTable[MAC::Z]);
    MAC::PadTable(g.xcv, g.centreTable[MAC::X]); MAC::PadTable(g.ycv, g.centreTable[MAC::Y]); MAC::PadTable(g.zcv, g.centreTable[MAC::Z]);
    MAC::GapTable(g.dxs, g.gapTable[MAC::X]);   MAC::GapTable(g.dys, g.gapTable[MAC::Y]);   MAC::GapTable(g.dzs, g.gapTable[MAC::Z]);
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.is2D ? 1 : g.Nz;
    g.cellVolume.resize((size_t)Nx * Ny * Nz);
    if (g.is2D)
    {
        for (int i = 0; i < Ny; i++)
            for (int j = 0; j < Nx; j++)
                g.cellVolume[(size_t)i * Nx + j] = g.Width(MAC::X, j) * g.Width(MAC::Y, i);
    }
    else
    {
        for (int i = 0; i < Ny; i++)
            for (int j = 0; j < Nx; j++)
                for (int k = 0; k < Nz; k++)
                    g.cellVolume[(size_t)i * (Nx * Nz) + j * Nz + k] = g.Width(MAC::X, j) * g.Width(MAC::Y, i) * g.Width(MAC::Z, k);
    }
    SIMULATION.spacing.nonUniform = true;
    SIMULATION.spacing.dx = g.dxs; SIMULATION.spacing.dy = g.dys; SIMULATION.spacing.dz = g.dzs;
    SIMULATION.spacing.xf = g.xfv; SIMULATION.spacing.yf = g.yfv; SIMULATION.spacing.zf = g.zfv;
    SIMULATION.spacing.xc = g.xcv; SIMULATION.spacing.yc = g.ycv; SIMULATION.spacing.zc = g.zcv;
    double hmin = 1e300;
    for (double d : g.dxs) hmin = std::min(hmin, d);
    for (double d : g.dys) hmin = std::min(hmin, d);
    if (!g.is2D) for (double d : g.dzs) hmin = std::min(hmin, d);
    g.dh = hmin;
    const size_t nu = g.is2D ? (size_t)(Nx + 1) * Ny : (size_t)(Nx + 1) * Ny * Nz;
    const size_t nv = g.is2D ? (size_t)Nx * (Ny + 1) : (size_t)Nx * (Ny + 1) * Nz;
    g.u = VectorXd::Zero(nu);
    g.v = VectorXd::Zero(nv);
    g.w = g.is2D ? VectorXd() : VectorXd::Zero((size_t)Nx * Ny * (Nz + 1));
    g.p = VectorXd::Zero((size_t)Nx * Ny * Nz);
    g.cellTypes.assign((size_t)Nx * Ny * Nz, (unsigned char)FLUID_CELL);
    g.boundaryListsStale = true;
    g.BuildStrides();
}

// Scheme 5: the reference's own boundary-condition replay on the case's fields, with the lists it built.
static int BoundaryReplay(MAC &grid, int dim, double time, const std::vector<double> &pIn, const char *out)
{
    if (dim == 3) grid.SetBoundaryFunctions(SIMULATION.VelocityBoundaryFunction, SIMULATION.PressureBoundaryFunction);
    else grid.SetBoundaryFunctions(SIMULATION.VelocityBoundaryFunction2D, SIMULATION.PressureBoundaryFunction2D);
    for (size_t c = 0; c < pIn.size(); c++) grid.p[c] = pIn[c];
    grid.EnforceVelocityBC(time);
    grid.EnforcePressureBC(time);

    FILE *o = std::fopen(out, "wb");
    if (!o) { std::fprintf(stderr, "cannot write %s\n", out); return 2; }
    std::fwrite("NBBC0001", 1, 8, o);
    const int32_t hdr[11] = {grid.Nx, grid.Ny, dim == 3 ? grid.Nz : 1, (int32_t)grid.solidFaceList[0].size(),
                             (int32_t)grid.solidFaceList[1].size(), (int32_t)grid.solidFaceList[2].size(),
                             (int32_t)grid.prescribedList.size(), (int32_t)grid.copyList.size(),
                             (int32_t)grid.ringList.size(), (int32_t)grid.inletFaces.size(),
                             (int32_t)grid.outflowFaces.size()};
    WriteN(o, hdr, 11);
    for (int c = 0; c < 3; c++)
    {
        std::vector<int32_t> v(grid.solidFaceList[c].begin(), grid.solidFaceList[c].end());
        WriteN(o, v.data(), v.size());
    }
    {
        const size_t n = grid.prescribedList.size();
        std::vector<int32_t> comp(n), index(n);
        std::vector<double> value(n);
        for (size_t q = 0; q < n; q++)
        {
            const MAC::PrescribedEntry &e = grid.prescribedList[q];
            comp[q] = (int32_t)e.c;
            index[q] = e.index;
            if (dim == 3)
            {
                const Vec3 vel = grid.boundaryVelocity3D(e.x, e.y, e.z, time);
                value[q] = e.c == MAC::U ? vel.u : (e.c == MAC::V ? vel.v : vel.w);
            }
            else
            {
                const Vec2 vel = grid.boundaryVelocity2D(e.x, e.y, time);
                value[q] = e.c == MAC::U ? vel.u : vel.v;
            }
        }
        WriteN(o, comp.data(), n); WriteN(o, index.data(), n); WriteN(o, value.data(), n);
    }
    {
        const size_t n = grid.copyList.size();
        std::vector<int32_t> comp(n), dst(n), src(n);
        for (size_t q = 0; q < n; q++)
        {
            comp[q] = (int32_t)grid.copyList[q].c; dst[q] = grid.copyList[q].dst; src[q] = grid.copyList[q].src;
        }
        WriteN(o, comp.data(), n); WriteN(o, dst.data(), n); WriteN(o, src.data(), n);
    }
    {
        const size_t n = grid.ringList.size();
        std::vector<int32_t> dst(n), kind(n), src(n);
        std::vector<double> value(n, 0.0);
        for (size_t q = 0; q < n; q++)
        {
            const MAC::RingEntry &e = grid.ringList[q];
            dst[q] = e.dst; kind[q] = e.kind; src[q] = e.src;
            if (e.kind == 1) value[q] = grid.PrescribedPressure(e.i, e.j, e.k, time);
        }
        WriteN(o, dst.data(), n); WriteN(o, kind.data(), n); WriteN(o, src.data(), n); WriteN(o, value.data(), n);
    }
    for (const std::vector<MAC::FluxFace> *faces : {&grid.inletFaces, &grid.outflowFaces})
    {
        const size_t n = faces->size();
        std::vector<int32_t> comp(n), index(n), outer(n);
        std::vector<double> area(n), sign(n);
        for (size_t q = 0; q < n; q++)
        {
            const MAC::FluxFace &e = (*faces)[q];
            comp[q] = (int32_t)e.c; index[q] = e.index; outer[q] = e.outer; area[q] = e.area; sign[q] = e.sign;
        }
        WriteN(o, comp.data(), n); WriteN(o, index.data(), n); WriteN(o, outer.data(), n);
        WriteN(o, area.data(), n); WriteN(o, sign.data(), n);
    }
    WriteN(o, grid.u.data(), grid.u.size());
    WriteN(o, grid.v.data(), grid.v.size());
    if (dim == 3) WriteN(o, grid.w.data(), grid.w.size());
    WriteN(o, grid.p.data(), grid.p.size());
    std::fclose(o);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc != 3) { std::fprintf(stderr, "usage: ref_harness case.bin result.bin\n"); return 2; }
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) { std::fprintf(stderr, "cannot open %s\n", argv[1]); return 2; }
    char magic[8];
    ReadN(f, magic, 8);
    if (std::memcmp(magic, "NBCASE01", 8) != 0) { std::fprintf(stderr, "bad magic\n"); return 2; }
    int32_t h[16];
    ReadN(f, h, 16);
    const int dim = h[0], gridMode = h[1], gridSize = h[2], labelMode = h[6], scheme = h[8];
    double dom[6], rho, dt, tol, time;
    ReadN(f, dom, 6); ReadN(f, &rho, 1); ReadN(f, &dt, 1); ReadN(f, &tol, 1); ReadN(f, &time, 1);
    std::vector<double> wx, wy, wz;
    if (gridMode == 1)
    {
        wx.resize(h[3]); wy.resize(h[4]); wz.resize(dim == 3 ? h[5] : 0);
        ReadN(f, wx.data(), wx.size()); ReadN(f, wy.data(), wy.size()); ReadN(f, wz.data(), wz.size());
    }

    DIMENSION = dim;
    RegisterHarnessMethod(h[12]);
    THREAD_COUNT = h[11] > 0 ? h[11] : 1;
    omp_set_num_threads(THREAD_COUNT);
    Eigen::setNbThreads(THREAD_COUNT);
    GPU_ACCELERATION = 0;
    ADAPTATIVE_TIMESTEP = 0;
    SIMULATION.domain = Domain{dom[0], dom[1], dom[2], dom[3], dom[4], dom[5]};
    SIMULATION.GRID_SIZE = gridSize;
    SIMULATION.RHO = rho;
    SIMULATION.dt = dt;
    SIMULATION.dtConfigured = dt;
    SIMULATION.time = time;
    SIMULATION.f = Vec3{0.0, 0.0, 0.0};
    SIMULATION.grid.nonUniform = (gridMode == 1);
    PRESSURE_SETTINGS.needsCompatibilityCondition = h[7] != 0;
    PRESSURE_SETTINGS.warmStart = scheme == 2;
    // The PRESSURE block the oracle runs with: eigen_* keys only (PressureSettings.h:212-255).
    {
        const char *solver = h[9] == 1 ? "AMG" : (h[9] == 2 ? "BICGSTAB" : "CG");
        char text[256];
        std::snprintf(text, sizeof(text), "eigen_solver=%s\neigen_preconditioner=DIAGONAL\neigen_tolerance=%.17g\neigen_max_iters=%d\n",
                      solver, tol, h[10]);
        PRESSURE_SETTINGS.text = text;
    }

    static MAC grid;
    grid = MAC();
    if (gridMode == 0)
        grid.InitializeGrid(SIMULATION.domain, dim == 2);
    else
        InitStretched(grid, dim, dom, wx, wy, wz);
    const int Nx = grid.Nx, Ny = grid.Ny, Nz = dim == 3 ? grid.Nz : 1;
    if (Nx != h[14] || Ny != h[15]) { std::fprintf(stderr, "grid size mismatch %d %d vs %d %d\n", Nx, Ny, h[14], h[15]); return 4; }
    SIMULATION.dh = grid.dh; SIMULATION.Nx = grid.Nx; SIMULATION.Ny = grid.Ny; SIMULATION.Nz = grid.Nz;
    SIMULATION.GRID_SOL = &grid; SIMULATION.GRID_ANT = &grid;
    const size_t cells = (size_t)Nx * Ny * Nz;

    if (labelMode == 0)
    {
        int32_t len = 0;
        ReadN(f, &len, 1);
        std::string text(len, '\0');
        ReadN(f, &text[0], len);
        if (!SCENE.LoadText(text)) { std::fprintf(stderr, "scene: %s\n", SCENE.error.c_str()); return 5; }
        SIMULATION.VelocityBoundaryFunction = SCENE_VELOCITY;
        SIMULATION.PressureBoundaryFunction = SCENE_PRESSURE;
        SIMULATION.VelocityBoundaryFunction2D = SCENE_VELOCITY_2D;
        SIMULATION.PressureBoundaryFunction2D = SCENE_PRESSURE_2D;
        SIMULATION.BoundaryKindFunction = SCENE_BOUNDARY_KIND;
        if (dim == 3) grid.SetSolidMask(SCENE_SOLID_MASK);
        else grid.SetSolidMask(SCENE_SOLID_MASK_2D);
    }
    else
    {
        std::vector<uint8_t> lab(cells);
        ReadN(f, lab.data(), cells);
        for (int i = 0; i < Ny; i++)
            for (int j = 0; j < Nx; j++)
                for (int k = 0; k < Nz; k++)
                {
                    if (dim == 3) grid.SetSolid(i, j, k, lab[((size_t)i * Nx + j) * Nz + k]);
                    else grid.SetSolid(i, j, lab[(size_t)i * Nx + j]);
                }
    }
    grid.u.setZero(); grid.v.setZero(); grid.p.setZero();
    if (dim == 3) grid.w.setZero();
    ReadN(f, grid.u.data(), grid.u.size());
    ReadN(f, grid.v.data(), grid.v.size());
    if (dim == 3) ReadN(f, grid.w.data(), grid.w.size());
    // the previous step: the same geometry and labels, its own pressure
    static MAC gridAnt;
    MAC *ant = nullptr;
    if (scheme == 1 || scheme == 2)
    {
        gridAnt = grid;
        ReadN(f, gridAnt.p.data(), gridAnt.p.size());
        ant = &gridAnt;
    }
    std::vector<double> pBC;
    if (scheme == 5)
    {
        pBC.resize(grid.p.size());
        ReadN(f, pBC.data(), pBC.size());
    }
    std::vector<uint8_t> typesBefore;
    double origin[3] = {0.0, 0.0, 0.0};
    if (scheme == 4)
    {
        int64_t np = 0;
        ReadN(f, &np, 1);
        std::vector<double> xyz((size_t)np * 3);
        ReadN(f, xyz.data(), xyz.size());
        static ParticleSet particles;
        particles.data.assign((size_t)np, Particle{});
        particles.count = (int)np;
        for (int64_t q = 0; q < np; q++)
        {
            particles.data[q].isActive = true;
            particles.data[q].x = xyz[3 * q];
            particles.data[q].y = xyz[3 * q + 1];
            particles.data[q].z = xyz[3 * q + 2];
        }
        typesBefore.assign(grid.cellTypes.data(), grid.cellTypes.data() + cells);
        origin[0] = grid.FacePos(MAC::X, 0);
        origin[1] = grid.FacePos(MAC::Y, 0);
        origin[2] = dim == 3 ? grid.FacePos(MAC::Z, 0) : 0.0;
        if (dim == 3) FLIP3D::UpdateFluidCells(&grid, &particles);
        else FLIP2D::UpdateFluidCells(&grid, &particles);
    }
    std::fclose(f);
    if (scheme == 5) return BoundaryReplay(grid, dim, time, pBC, argv[2]);

    // The pressure ring as the step sees it (SolveScheme's first call, PressureSolver3D.cpp:281).
    grid.EnforcePressureBC(time);

    const double t0 = Now();
    const PressureScheme ps = scheme == 1 ? PRESSURE_INCREMENTAL : PRESSURE_CHORIN;
    if (dim == 3) PressureSolver3D::InitializePressureSolver(&grid, ps);
    else PressureSolver2D::InitializePressureSolver(&grid, ps);
    const double tAssemble = Now() - t0;
    MAC *old = scheme == 1 ? ant : nullptr; // DirichletSum's `old` under the incremental scheme

    PressureSystem &S = dim == 3 ? PressureSolver3D::SYSTEM : PressureSolver2D::SYSTEM;
    const std::vector<int> &IDP = dim == 3 ? PressureSolver3D::IDP : PressureSolver2D::IDP;
    const int n = (int)S.A.rows();

    // The right-hand side, formed with the reference's own accessors in SolveScheme's expression order
    // (PressureSolver3D.cpp:288-307, PressureSolver2D.cpp:263-280).
    std::vector<double> braw(n, 0.0), b(n, 0.0);
    {
        const double scale = grid.nonUniform ? 1.0 : 1.0 / (grid.dh * grid.dh);
        const double rhoDt = SIMULATION.RHO / SIMULATION.dt;
        for (int i = 1; i < Ny - 1; i++)
            for (int j = 1; j < Nx - 1; j++)
                for (int k = (dim == 3 ? 1 : 0); k < (dim == 3 ? Nz - 1 : 1); k++)
                {
                    const int id = IDP[((size_t)i * Nx + j) * Nz + k];
                    if (id < 0) continue;
                    if (dim == 3)
                        braw[id] = rhoDt * grid.GetDivergencyAt(i, j, k) * (grid.nonUniform ? grid.CellVolume(i, j, k) : 1.0)
                                   - scale * PressureSolver3D::DirichletSum(&grid, old, i, j, k);
                    else
                        braw[id] = rhoDt * grid.GetDivergencyAt(i, j) * (grid.nonUniform ? grid.CellVolume(i, j) : 1.0)
                                   - scale * PressureSolver2D::DirichletSum(&grid, old, i, j);
                }
        b = braw;
        if (PRESSURE_SETTINGS.needsCompatibilityCondition && S.singular && n > 0)
        {
            double mean = 0.0;
            for (int q = 0; q < n; q++) mean += b[q];
            mean /= n;
            for (int q = 0; q < n; q++) b[q] -= mean;
            SubtractMean(b.data(), n);
        }
    }

    double refNorm = 0.0;
    if (scheme == 1 && n > 0)
    {
        Eigen::Map<const Eigen::VectorXd> bv(b.data(), n);
        refNorm = dim == 3 ? PressureSolver3D::IncrementReferenceNorm(ant, bv)
                           : PressureSolver2D::IncrementReferenceNorm(ant, bv);
    }

    // Cold solve (AMGCL builds its hierarchy here), then warm repeats of the same solve (Chorin only).
    double t1 = Now();
    int iters = -1;
    if (scheme == 3)
    {
        // Explicit2D::Pressure enforces the ring at its time + dt, so it is handed time - dt
        EXPLICIT_SETTINGS.tolerance = tol;
        EXPLICIT_SETTINGS.maxIterations = h[10];
        Explicit2D::Pressure(nullptr, &grid, nullptr, time - SIMULATION.dt);
    }
    else
    {
        if (dim == 3) PressureSolver3D::SolvePressure(ant, &grid, nullptr, time);
        else PressureSolver2D::SolvePressure(ant, &grid, nullptr, time);
        iters = PRESSURE_TELEMETRY.lastIterations;
    }
    const double tCold = Now() - t1;
    const int repeats = scheme == 0 ? h[13] : 0;
    double tWarm = 0.0;
    std::vector<double> tEach(repeats > 0 ? repeats : 0);
    for (int r = 0; r < repeats; r++)
    {
        t1 = Now();
        if (dim == 3) PressureSolver3D::SolvePressure(nullptr, &grid, nullptr, time);
        else PressureSolver2D::SolvePressure(nullptr, &grid, nullptr, time);
        tEach[r] = Now() - t1;
        tWarm += tEach[r];
    }
    if (repeats > 0) tWarm /= repeats;

    std::vector<double> x(n, 0.0);
    for (size_t c = 0; c < cells; c++)
        if (IDP[c] >= 0) x[IDP[c]] = grid.p[c];
    std::vector<double> pAfter(grid.p.data(), grid.p.data() + grid.p.size());

    double relres = 0.0;
    if (n > 0)
    {
        Eigen::Map<const Eigen::VectorXd> xv(x.data(), n), bv(b.data(), n);
        const double bn = bv.norm();
        relres = bn > 0 ? (bv - S.A * xv).norm() / bn : 0.0;
    }

    t1 = Now();
    if (scheme == 3) Explicit2D::Projection(nullptr, &grid, nullptr, time);
    else if (dim == 3) PressureSolver3D::ProjectPressure(&grid);
    else PressureSolver2D::ProjectPressure(&grid);
    const double tProject = Now() - t1;
    if (scheme == 1) // the rest of Project under the incremental scheme
    {
        if (dim == 3) PressureSolver3D::AccumulatePressureIncrement(ant, &grid);
        else PressureSolver2D::AccumulatePressureIncrement(ant, &grid);
    }

    // Post-projection divergence over FLUID cells (MAC::GetDivergencyAt).
    double maxDiv = 0.0;
    for (int i = 1; i < Ny - 1; i++)
        for (int j = 1; j < Nx - 1; j++)
            for (int k = (dim == 3 ? 1 : 0); k < (dim == 3 ? Nz - 1 : 1); k++)
            {
                const double d = dim == 3 ? grid.GetDivergencyAt(i, j, k) : grid.GetDivergencyAt(i, j);
                maxDiv = std::max(maxDiv, std::fabs(d));
            }

    // NB_REF_LEAN=1 (large grids): the labels, numbering, matrix and right-hand sides are left out of the result
    // (flag 1 in the last double of the header); x, p, the fields, the tables and the times stay
    const char *leanEnv = std::getenv("NB_REF_LEAN");
    const bool lean = leanEnv && leanEnv[0] == '1';
    FILE *o = std::fopen(argv[2], "wb");
    if (!o) { std::fprintf(stderr, "cannot write %s\n", argv[2]); return 2; }
    std::fwrite("NBRES001", 1, 8, o);
    const int32_t nnz = (int32_t)S.A.nonZeros();
    const int32_t oh[8] = {Nx, Ny, Nz, n, lean ? 0 : nnz, iters, S.singular ? 1 : 0, THREAD_COUNT};
    WriteN(o, oh, 8);
    const double od[8] = {tAssemble, tCold, tWarm, tProject, relres, maxDiv, grid.dh, lean ? 1.0 : 0.0};
    WriteN(o, od, 8);
    if (!lean)
    {
        WriteN(o, grid.cellTypes.data(), cells);
        std::vector<int32_t> idp(IDP.begin(), IDP.end());
        WriteN(o, idp.data(), cells);
        std::vector<int32_t> rp(n + 1), cl(nnz);
        for (int r = 0; r <= n; r++) rp[r] = S.A.outerIndexPtr()[r];
        for (int q = 0; q < nnz; q++) cl[q] = S.A.innerIndexPtr()[q];
        WriteN(o, rp.data(), n + 1);
        WriteN(o, cl.data(), nnz);
        WriteN(o, S.A.valuePtr(), nnz);
        WriteN(o, braw.data(), n);
        WriteN(o, b.data(), n);
    }
    WriteN(o, x.data(), n);
    WriteN(o, pAfter.data(), pAfter.size());
    WriteN(o, grid.u.data(), grid.u.size());
    WriteN(o, grid.v.data(), grid.v.size());
    if (dim == 3) WriteN(o, grid.w.data(), grid.w.size());
    for (int a = 0; a < 3; a++)
    {
        const int32_t nw = (int32_t)grid.widthTable[a].size(), ng = (int32_t)grid.gapTable[a].size();
        WriteN(o, &nw, 1); WriteN(o, grid.widthTable[a].data(), nw);
        WriteN(o, &ng, 1); WriteN(o, grid.gapTable[a].data(), ng);
        const int32_t nc = (int32_t)grid.centreTable[a].size();
        WriteN(o, &nc, 1); WriteN(o, grid.centreTable[a].data(), nc);
    }
    const int32_t nr = (int32_t)tEach.size();
    WriteN(o, &nr, 1);
    WriteN(o, tEach.data(), tEach.size());
    if (scheme == 1 || scheme == 2)
    {
        WriteN(o, &refNorm, 1);
        WriteN(o, grid.p.data(), grid.p.size());
    }
    if (scheme == 4)
    {
        WriteN(o, origin, 3);
        WriteN(o, typesBefore.data(), cells);
    }
    std::fclose(o);
    return 0;
}
