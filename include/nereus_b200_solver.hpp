// nereus_b200_solver.hpp -- C++ host side of the B200 pressure projection, shaped like the reference's
// PressureSolver3D / PressureSolver2D static classes (src/Methods/PPESolver/PressureSolver3D.h:49-75) so that a NEREUS
// build can route its pressure step through include/nereus_b200.h with the same calls, argument meaning and error
// behaviour. Header-only; link with nereus_cfd_b200/libnereus_b200.so.
//
// The grid is passed as a view of the MAC's arrays (src/headers/Core/MAC.h:424-448): sizes with the ring, the cell
// types, the padded Width / FaceGap tables and the four fields, all host memory owned by the caller.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "nereus_b200.h"

namespace nereus_b200
{

// What the pressure step reads and writes of a MAC grid.
struct GridView
{
    int dim = 3;
    int Nx = 0, Ny = 0, Nz = 1;     // ring included; Nz = 1 in 2D
    bool nonUniform = false;
    double dh = 0.0;                // MAC::dh (the uniform cell size)
    const uint8_t *cellTypes = nullptr;
    const double *width[3] = {nullptr, nullptr, nullptr}; // padded Width tables, N + 2 entries
    const double *gap[3] = {nullptr, nullptr, nullptr};   // padded FaceGap tables, N + 1 entries
    double *u = nullptr, *v = nullptr, *w = nullptr, *p = nullptr;
};

struct Error : std::runtime_error
{
    int status;
    Error(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};

inline void Check(int status)
{
    if (status != NB_OK && status != NB_NOT_CONVERGED) throw Error(status, nereus_b200_last_error());
}

// One pressure system on one GPU, the role the reference's static SYSTEM/IDP play per dimension.
class PressureSolver
{
  public:
    explicit PressureSolver(int precision = NB_PRECISION_MIXED, int device = 0)
    {
        nereus_b200_default_options(&opt_);
        opt_.precision = precision;
        opt_.use_graphs = 1;
        opt_.device = device;
    }
    ~PressureSolver() { DestroyPressureSolver(); }
    PressureSolver(const PressureSolver &) = delete;
    PressureSolver &operator=(const PressureSolver &) = delete;

    nb_options &Options() { return opt_; }

    // InitializePressureSolver (PressureSolver3D.cpp:89-102): backend up, system assembled for this layout, the
    // scheme (SYSTEM.scheme) kept for SolvePressure. warmStart: PRESSURE_SETTINGS.warmStart for the Chorin scheme.
    void InitializePressureSolver(const GridView &g, int scheme = NB_SCHEME_CHORIN, bool warmStart = false)
    {
        if (scheme != NB_SCHEME_CHORIN && scheme != NB_SCHEME_INCREMENTAL) throw Error(NB_BAD_INPUT, "unknown scheme");
        scheme_ = scheme;
        warmStart_ = warmStart;
        if (!ctx_) Check(nereus_b200_create(&ctx_, &opt_));
        EnsureSystem(g);
    }

    // EnsureSystem (PressureSolver3D.cpp:120-124): the library rebuilds only when the cell types changed.
    void EnsureSystem(const GridView &g)
    {
        Check(nereus_b200_set_layout(ctx_, g.dim, g.Nx, g.Ny, g.dim == 3 ? g.Nz : 1, g.cellTypes, g.width, g.gap,
                                     g.nonUniform ? 1 : 0, g.dh));
    }

    void DestroyPressureSolver()
    {
        if (ctx_) nereus_b200_destroy(ctx_);
        ctx_ = nullptr;
    }
    void ReleasePressureSolver() { DestroyPressureSolver(); }

    // SolvePressure (PressureSolver3D.cpp:279-345) fused with Project (:396-438) in the initialised scheme: p must
    // carry the ring values EnforcePressureBC(time) wrote; pPrev is gridAnt's pressure (required by the incremental
    // scheme, the guess of the Chorin warm start, else may be null). Returns the report; NOT_CONVERGED is reported,
    // not thrown.
    nb_result SolvePressure(const GridView &g, double rho, double dt, bool needsCompat, double tol,
                            const double *pPrev = nullptr)
    {
        EnsureSystem(g);
        nb_result r{};
        if (scheme_ == NB_SCHEME_INCREMENTAL || (warmStart_ && pPrev))
            Check(nereus_b200_project_ex(ctx_, g.u, g.v, g.w, g.p, pPrev, rho, dt, scheme_, needsCompat ? 1 : 0,
                                         warmStart_ ? 1 : 0, tol, &r));
        else
            Check(nereus_b200_project(ctx_, g.u, g.v, g.w, g.p, rho, dt, NB_SCHEME_CHORIN, needsCompat ? 1 : 0, tol,
                                      &r));
        lastIterations_ = r.iters_inner;
        return r;
    }

    // SolveIncremental + Project (PressureSolver3D.h:58,71) from the previous step's pressure, whatever the
    // initialised scheme.
    nb_result SolveIncremental(const double *pPrev, const GridView &g, double rho, double dt, bool needsCompat,
                               double tol)
    {
        EnsureSystem(g);
        nb_result r{};
        Check(nereus_b200_project_ex(ctx_, g.u, g.v, g.w, g.p, pPrev, rho, dt, NB_SCHEME_INCREMENTAL,
                                     needsCompat ? 1 : 0, 0, tol, &r));
        lastIterations_ = r.iters_inner;
        return r;
    }

    // The two registered steps separately, for a caller that keeps them apart.
    nb_result SolvePressureOnly(const GridView &g, double rho, double dt, bool needsCompat, double tol)
    {
        EnsureSystem(g);
        nb_result r{};
        Check(nereus_b200_solve_pressure(ctx_, g.u, g.v, g.w, g.p, rho, dt, NB_SCHEME_CHORIN, needsCompat ? 1 : 0,
                                         tol, &r));
        lastIterations_ = r.iters_inner;
        return r;
    }
    void ProjectPressure(const GridView &g, double rho, double dt)
    {
        Check(nereus_b200_project_velocity(ctx_, g.u, g.v, g.w, g.p, rho, dt));
    }

    // SolveLaplacian (PressureSolver3D.cpp:355-371): false when f's size is not SystemSize().
    bool SolveLaplacian(const GridView &g, const std::vector<double> &f, std::vector<double> &x, double tol = 1e-12)
    {
        EnsureSystem(g);
        const int n = SystemSize();
        if (n == 0 || (int)f.size() != n) return false;
        x.assign(n, 0.0);
        nb_result r{};
        Check(nereus_b200_solve_laplacian(ctx_, f.data(), x.data(), tol, &r));
        return true;
    }

    int SystemSize() const { return ctx_ ? nereus_b200_system_size(ctx_) : 0; }
    int LastIterations() const { return lastIterations_; }

    // GetIDP for every cell at once: idp holds Nx*Ny*Nz entries, -1 off the system.
    void GetIDP(int32_t *idp) { Check(nereus_b200_get_idp(ctx_, idp)); }

  private:
    nb_options opt_{};
    nb_ctx *ctx_ = nullptr;
    int lastIterations_ = 0;
    int scheme_ = NB_SCHEME_CHORIN;
    bool warmStart_ = false;
};

// FLIP3D::UpdateFluidCells / FLIP2D::UpdateFluidCells (src/Methods/FLIP/FLIP3D.cpp:784-833,
// src/Methods/FLIP/FLIP2D.cpp:648-691) on host labels, in place. x0 points at the first particle's x with y and z the
// next two doubles, rows `stride` doubles apart: the reference's Particle array is &particles->data[0].x, stride 7.
// origin = FacePos(X|Y|Z, 0) (origin[2] unread in 2D), dh = SIMULATION.dh. Returns the number of particles skipped
// as outside the labels (the reference would index outside them).
inline int64_t UpdateFluidCells(int dim, int Nx, int Ny, int Nz, const double origin[3], double dh, const double *x0,
                                int64_t count, int64_t stride, uint8_t *cellTypes)
{
    int64_t skipped = 0;
    const double *y0 = x0 ? x0 + 1 : nullptr, *z0 = (x0 && dim == 3) ? x0 + 2 : nullptr;
    const int st = nereus_b200_update_fluid_cells(dim, Nx, Ny, Nz, origin[0], origin[1], dim == 3 ? origin[2] : 0.0,
                                                  dh, x0, y0, z0, count, stride, cellTypes, &skipped);
    if (st != NB_OK) throw Error(st, nereus_b200_last_error());
    return skipped;
}

// MAC::EnforceVelocityBC and MAC::EnforcePressureBC (src/MAC.cpp:811-865) on device fields, from the lists
// MAC::BuildBoundaryLists made (rebuild the object when the MAC rebuilds them). The calls queue work on `stream`.
class BoundaryReplay
{
  public:
    BoundaryReplay(int device, const nb_bc_lists &lists)
    {
        const int st = nereus_b200_bc_create(device, &lists, &bc_);
        if (st != NB_OK) throw Error(st, nereus_b200_last_error());
    }
    ~BoundaryReplay() { nereus_b200_bc_destroy(bc_); }
    BoundaryReplay(const BoundaryReplay &) = delete;
    BoundaryReplay &operator=(const BoundaryReplay &) = delete;

    // prescValues: the boundary velocity function at each prescribedList entry (device), or null without one.
    void EnforceVelocityBC(double *u, double *v, double *w, const double *prescValues, void *stream = nullptr)
    {
        const int st = nereus_b200_bc_enforce_velocity(bc_, u, v, w, prescValues, stream);
        if (st != NB_OK) throw Error(st, nereus_b200_last_error());
    }
    // ringValues: PrescribedPressure at each ringList entry of kind 1 (device), or null for 0 there.
    void EnforcePressureBC(double *p, const double *ringValues, void *stream = nullptr)
    {
        const int st = nereus_b200_bc_enforce_pressure(bc_, p, ringValues, stream);
        if (st != NB_OK) throw Error(st, nereus_b200_last_error());
    }
    int VelocityLevels() const { return Levels(0); }
    int PressureLevels() const { return Levels(1); }

  private:
    int Levels(int pressure) const
    {
        int v = 0, p = 0;
        nereus_b200_bc_levels(bc_, &v, &p);
        return pressure ? p : v;
    }
    nb_bc *bc_ = nullptr;
};

// Many pressure systems of one grid shape stepped together (nereus_b200_batch_*): where the reference makes one
// SolvePressureSystem call per system (src/Methods/PPESolver/PressureSettings.h:578-624), slot i of a batch holds
// system i's layout and one Project call runs the Chorin step of slots 0 .. n-1 on their device fields. A system's
// result does not depend on the rest of the batch, and agrees with a PressureSolver's within the solve's tolerance.
class BatchSolver
{
  public:
    explicit BatchSolver(int capacity, int device = 0, bool autotune = true)
    {
        nb_options o;
        nereus_b200_default_options(&o);
        o.device = device;
        o.autotune = autotune ? 1 : 0;
        const int st = nereus_b200_batch_create(&b_, &o, capacity);
        if (st != NB_OK) throw Error(st, nereus_b200_last_error());
    }
    ~BatchSolver() { nereus_b200_batch_destroy(b_); }
    BatchSolver(const BatchSolver &) = delete;
    BatchSolver &operator=(const BatchSolver &) = delete;

    // the layout of slot i (unchanged bytes keep its hierarchy, as PressureLayoutChanged)
    void SetLayout(int slot, const GridView &g)
    {
        Check(nereus_b200_batch_set_layout(b_, slot, g.dim, g.Nx, g.Ny, g.Nz, g.cellTypes, g.width, g.gap,
                                           g.nonUniform ? 1 : 0, g.dh));
    }
    // the step of slots 0 .. items.size()-1; results[i] is slot i's report
    void Project(const std::vector<nb_batch_item> &items, std::vector<nb_result> &results)
    {
        results.assign(items.size(), nb_result{});
        Check(nereus_b200_batch_project_device(b_, (int)items.size(), items.data(), results.data()));
    }

  private:
    nb_batch *b_ = nullptr;
};

} // namespace nereus_b200
