/*
 * nereus_b200.h -- the C ABI of the B200 pressure projection for NEREUS (RaphaelLaroca/NEREUS_CFD).
 *
 * It replaces the pressure step of the reference's PressureSolver2D / PressureSolver3D static classes
 * (src/Methods/PPESolver/PressureSolver3D.h:49-75, PressureSolver2D.h:49-76): the divergence of the intermediate MAC
 * face velocities, the Poisson system from the cell types and the (stretched) spacing tables, the solve, the
 * constant level, the scatter and pressure ring, and the pressure-gradient velocity correction. One context serves
 * one grid on one GPU; a batch and a serving queue advance many independent grids at once.
 *
 * Conventions
 *   - Status codes (nb_status): 0 OK; no exception crosses the ABI.
 *   - Fields are the MAC grid's (src/headers/Core/MAC.h:235-254, 369-374): cell (i,j,k) = (y,x,z) at
 *     (i*Nx + j)*Nz + k, u with Nx+1 entries along x, v with Ny+1 along y, w with Nz+1 along z; Nx, Ny, Nz include
 *     the one-cell border ring. In 2D pass Nz = 1 and w = NULL.
 *   - Spacing tables are the reference's padded ones (MAC.h:439-448): width[a] has N_a + 2 entries
 *     (width[a][n+1] = Width(a, n), n = -1..N_a), gap[a] has N_a + 1 (gap[a][n+1] = FaceGap(a, n), n = -1..N_a-1).
 *     In 2D width[2]/gap[2] describe the single z cell and are not read.
 *   - Host pointers unless the function name says _device. The library allocates its own device memory; it is not
 *     reentrant across host threads for one context (one context per host thread, as the reference's statics are
 *     one system per dimension).
 */
#ifndef NEREUS_B200_H
#define NEREUS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum nb_status
{
    NB_OK = 0,
    NB_NOT_CONVERGED = 1, /* the solve hit its iteration caps; the result still holds the last iterate */
    NB_BAD_INPUT = 2,     /* sizes, pointers, tables or cell types the call cannot take */
    NB_OUT_OF_MEMORY = 3, /* device allocation failed, or a request exceeds the serving budget */
    NB_DEVICE_ERROR = 4,  /* a CUDA call failed; nb_last_error() says which */
    NB_NO_DEVICE = 5,     /* no CUDA device, or the library was not built for it */
    NB_BUSY = 6           /* a serving slot/ticket is not ready yet */
} nb_status;

/* Cell types (src/headers/Core/Definitions.h:191-196). */
enum { NB_FLUID = 0, NB_SOLID = 1, NB_EMPTY = 2, NB_INFLOW = 3, NB_PRESSURE = 4, NB_OUTFLOW = 5 };

/* What solves: plain FP64 MG-PCG, or FP32 MG-PCG inside FP64 iterative refinement. */
enum { NB_PRECISION_FP64 = 0, NB_PRECISION_MIXED = 1 };

/* Pressure schemes (src/Methods/PPESolver/PressureSettings.h:260). */
enum { NB_SCHEME_CHORIN = 0, NB_SCHEME_INCREMENTAL = 1 };

typedef struct nb_options
{
    int device;          /* CUDA device ordinal */
    int precision;       /* NB_PRECISION_FP64 or NB_PRECISION_MIXED */
    int max_iters;       /* FP64: PCG iterations; mixed: inner PCG iterations per refinement step */
    int max_outer;       /* mixed: refinement steps */
    double inner_tol;    /* mixed: relative residual reduction asked of each inner solve; for a tolerance below
                            inner_tol^2 each inner solve is asked for sqrt(tolerance) instead (at least 1e-6), so
                            that two refinement passes reach it */
    int pre_sweeps;      /* red-black Gauss-Seidel sweeps before the coarse correction */
    int post_sweeps;     /* ... and after it */
    int coarse_sweeps;   /* symmetric sweep pairs on the coarsest level */
    int max_levels;      /* multigrid levels at most (>= 1) */
    void *stream;        /* cudaStream_t to launch on; NULL: the context makes its own */
    int use_graphs;      /* 2 (default): the mixed solve runs as one captured CUDA graph, WHILE nodes over the
                            refinement passes and the CG iterations whose conditions the device sets (one host
                            synchronisation per solve; the FP64 form: one per restart); 1: one captured graph per
                            CG iteration (V-cycle included), the loop on the host; 0: plain launches. Graphs are
                            captured from a layout's second solve on: the first solve after a change of shape
                            launches plainly (capturing costs more than it saves once). All give the same result */
    int transfer_kernels; /* the restriction of colour-split levels: 0 (default): one thread per 4 coarse cells
                             where the coarse level has at least 2^20 cells, else one thread per coarse cell (a
                             batch: per 4 everywhere); 1: one thread per coarse cell everywhere; 2: one thread per 4
                             coarse cells everywhere. All three give the same result in a single solve */
    int pair_kernels;    /* FP32 kernels of the mixed form on 3D levels with Nz even (uniform or stretched):
                            2 (default): the colour-split layout, red and black cells in separate arrays, so that
                            one colour's sweep moves half the bytes; 1: cell pairs in the grid layout; 0: the
                            general per-cell kernels */
    int tail_cells;      /* the coarse end runs in one thread block from the first level with at most this many
                            cells (and shared memory for all of them); 0: no such block */
    int stretched_sweeps; /* red-black sweeps before and after the coarse correction on a stretched grid's levels
                             (their anisotropy asks for more smoothing); pre_sweeps/post_sweeps apply to uniform ones */
    int autotune;        /* batches: 1 (default): the launch shapes of the smoothing, residual and transfer kernels
                            are timed on the batch's first step and the fastest kept (cached per grid, level, kernel
                            and capacity); 0: the shapes a single solve takes. Neither changes a result */
    int skip_idle_tiles; /* 1 (default): on colour-split levels a block whose cells hold no unknown (the air of a
                            free-surface tank, a solid) skips its loads and stores; 0: every block works. Both give the
                            same result */
    int x_groups;        /* stretched 3D grids: 1 (default): coarsening pairs two x cells only where the pair is at
                            most 1.5 times as wide as a coarse y/z cell, and keeps the others whole, on every level
                            above the coarse end (the coarse cells stay near cubes, so point smoothing holds on
                            strongly stretched x); 0: every axis coarsened by two. y and z are always coarsened by
                            two. The iteration counts differ, the tolerance is met either way */
} nb_options;

typedef struct nb_result
{
    int status;          /* nb_status of the solve */
    int n;               /* unknowns: interior FLUID cells (SystemSize) */
    int singular;        /* no Dirichlet neighbour anywhere */
    int iters_outer;     /* refinement steps (mixed) or 1 (FP64) */
    int iters_inner;     /* PCG iterations summed over all steps (LastIterations) */
    int levels;          /* multigrid levels used */
    double b_norm;       /* ||b||_2 after the compatibility step */
    double rel_res;      /* ||b - A x||_2 / ||b||_2 in FP64, A the reference's matrix */
    double max_div;      /* max |div u| over FLUID cells after the projection (-1 when not computed) */
    double seconds;      /* device time of the call's solve + projection (CUDA events) */
    double latency_ms;   /* served requests: submission to completion on the host clock; 0 elsewhere */
} nb_result;

typedef struct nb_ctx nb_ctx;

/* ---- library ---- */
void nereus_b200_default_options(nb_options *opt);
const char *nereus_b200_last_error(void);
int nereus_b200_device_count(void);

/* ---- context: replaces PressureSolver3D::InitializePressureSolver / DestroyPressureSolver / ReleasePressureSolver
 *      (PressureSolver3D.h:52-54; PressureSolver3D.cpp:89-116) ---- */
int nereus_b200_create(nb_ctx **ctx, const nb_options *opt);
void nereus_b200_destroy(nb_ctx *ctx);

/* The grid's layout: cell types and spacing tables. Replaces EnsureSystem / AssembleSystem
 * (PressureSolver3D.cpp:120-178) and, like PressureLayoutChanged (PressureSettings.h:300-303), rebuilds the
 * hierarchy only when the sizes or the cell-type bytes differ from the last call. dh is the uniform cell size
 * (MAC::dh); nonUniform selects the stretched coefficients A_f/d_f (MatrixScale3D, PressureSolver3D.cpp:34-37). */
int nereus_b200_set_layout(nb_ctx *ctx, int dim, int Nx, int Ny, int Nz, const uint8_t *cellTypes,
                           const double *const width[3], const double *const gap[3], int nonUniform, double dh);

/* The pressure step and the projection on host fields, in place: SolveChorin/SolvePressure followed by
 * ProjectPressure (PressureSolver3D.cpp:279-345, 396-438). p carries the ring values MAC::EnforcePressureBC
 * wrote on the host (prescribed PRESSURE cells); the call replays the rest of the ring (EMPTY 0, others copied)
 * after the scatter, levels a singular system's mean to 0 when needsCompat is set, and corrects u, v, w on every
 * face with no solid side. tol: relative residual ||b - A x|| / ||b||. scheme must be NB_SCHEME_CHORIN. */
int nereus_b200_project(nb_ctx *ctx, double *u, double *v, double *w, double *p, double rho, double dt, int scheme,
                        int needsCompat, double tol, nb_result *out);

/* The reference's two registered steps separately. nereus_b200_solve_pressure is the "pressure" step alone
 * (SolveScheme, PressureSolver3D.cpp:279-328): p is written (unknowns scattered, ring replayed), u, v, w are only
 * read. nereus_b200_project_velocity is the "projection" step alone (ProjectPressure, PressureSolver3D.cpp:417-438)
 * with the pressure p as given. Running the two in turn gives what nereus_b200_project gives. */
int nereus_b200_solve_pressure(nb_ctx *ctx, const double *u, const double *v, const double *w, double *p, double rho,
                               double dt, int scheme, int needsCompat, double tol, nb_result *out);
int nereus_b200_project_velocity(nb_ctx *ctx, double *u, double *v, double *w, const double *p, double rho,
                                 double dt);

/* The same on fields already in device memory (sizes as above), in place; launches on the context's stream. */
int nereus_b200_project_device(nb_ctx *ctx, double *d_u, double *d_v, double *d_w, double *d_p, double rho,
                               double dt, int needsCompat, double tol, nb_result *out);

/* The pressure step with the previous step's pressure p_prev (the reference's gridAnt->p, ring included), then the
 * projection. Replaces SolveIncremental + Project (PressureSolver3D.h:58,71; PressureSolver3D.cpp:262-401) for
 * scheme = NB_SCHEME_INCREMENTAL: the solve is for phi = p^{n+1} - p^n with the prescribed-pressure increments
 * p_b(t^{n+1}) - p_b(t^n) on the ring, to ||r|| < tol max(||b||, ||b + A p^n||); the velocity is corrected with
 * grad phi; p returns as p^n + phi on the unknowns, levelled like LevelPressure, with p's prescribed ring values (as
 * given on entry) put back. For NB_SCHEME_CHORIN, warm_start = 1 starts the solve from p_prev on the unknowns
 * (BuildWarmStartGuess, PressureSolver3D.cpp:222-244; uniform grids only, as WarmStartEnabled); otherwise it is
 * nereus_b200_project. p_prev may be NULL for a cold Chorin step. Host buffers; the _device form takes device
 * pointers on the context's device and stream. */
int nereus_b200_project_ex(nb_ctx *ctx, double *u, double *v, double *w, double *p, const double *p_prev, double rho,
                           double dt, int scheme, int needs_compat, int warm_start, double tol, nb_result *out);
int nereus_b200_project_device_ex(nb_ctx *ctx, double *d_u, double *d_v, double *d_w, double *d_p,
                                  const double *d_p_prev, double rho, double dt, int scheme, int needs_compat,
                                  int warm_start, double tol, nb_result *out);

/* SolveLaplacian (PressureSolver3D.h:64, PressureSolver3D.cpp:355-371): L x = f on the unknowns, f and x indexed
 * like the matrix (IDP order, n = SystemSize entries); x = 0 at air and pressure cells, no flux at solids. */
int nereus_b200_solve_laplacian(nb_ctx *ctx, const double *f, double *x, double tol, nb_result *out);

/* SystemSize / LastIterations / GetIDP (PressureSolver3D.h:66-68, 75). idp: Nx*Ny*Nz entries, -1 off the system. */
int nereus_b200_system_size(const nb_ctx *ctx);
int nereus_b200_last_iterations(const nb_ctx *ctx);
int nereus_b200_get_idp(nb_ctx *ctx, int32_t *idp);

/* The assembled matrix as the reference's CSR (PressureSolver3D.cpp:128-178 + Eigen setFromTriplets): rows in IDP
 * order, ascending columns, the diagonal only when non-zero; computed on the device by the same coefficient code
 * the solver applies. rowptr: n+1 entries; col/val: up to 7n (3D) or 5n (2D). *nnz receives the count. */
int nereus_b200_export_matrix(nb_ctx *ctx, int32_t *rowptr, int32_t *col, double *val, int *nnz, int *singular);

/* The right-hand side before the compatibility step (PressureSolver3D.cpp:288-298), in IDP order, from host fields
 * (p carries the prescribed ring values; the ring is replayed first, as SolveScheme's EnforcePressureBC does). */
int nereus_b200_rhs(nb_ctx *ctx, const double *u, const double *v, const double *w, const double *p, double rho,
                    double dt, double *b);

/* ---- measurement (the reference's per-step wall times, SimulationManager.h:343-353, at kernel granularity) ----
 * With profiling on, the context brackets every launch of the selected kernels with CUDA events on its stream and
 * keeps, per kernel, the launch count, the summed device time and the algorithmic bytes one launch must move
 * (each array touched once). Kernel ids: */
enum
{
    NB_K_SMOOTH0 = 0,   /* red-black Gauss-Seidel half-sweep on the finest level */
    NB_K_RESIDUAL0 = 1, /* multigrid residual on the finest level */
    NB_K_RESTRICT0 = 2, /* restriction from the finest level */
    NB_K_PROLONG0 = 3,  /* prolongation + correction onto the finest level */
    NB_K_PAPPLY = 4,    /* CG direction update fused with the stencil apply and p.Ap */
    NB_K_XR = 5,        /* CG x, r update fused with r.r */
    NB_K_DOT = 6,       /* r.z */
    NB_K_REFINE = 7,    /* FP64 residual of the reference's matrix (+ correction in refinement) */
    NB_K_RHS = 8,       /* divergence / right-hand side */
    NB_K_PROJECT = 9,   /* velocity correction */
    NB_K_COARSE = 10,   /* every kernel on the coarser levels */
    NB_K_COUNT = 11
};
int nereus_b200_profile_enable(nb_ctx *ctx, unsigned kernelMask); /* bit k selects kernel id k; 0 turns it off */
int nereus_b200_profile_read(nb_ctx *ctx, int kernelId, int *launches, double *totalMs, double *bytesPerLaunch);
/* Kernel launches this library has made in this process (all contexts). */
long long nereus_b200_kernel_launches(void);

/* ---- scene labelling (Scene::CellTypeAt, src/headers/Core/Scene.h:639-686) on the device ---- */
enum { NB_PRIM_BOX = 0, NB_PRIM_SPHERE = 1, NB_PRIM_CYLINDER = 2, NB_PRIM_PLANE = 3 };
enum { NB_REGION_SOLID = 0, NB_REGION_FLUID = 1, NB_REGION_EMPTY = 2 };
enum { NB_BC_NOSLIP = 0, NB_BC_SLIP, NB_BC_MOVING, NB_BC_INLET, NB_BC_PRESSURE_OUTLET, NB_BC_OUTFLOW };

typedef struct nb_region
{
    int kind, region, axis, invert;
    double p0[3], p1[3], radius;
} nb_region;

typedef struct nb_scene
{
    int face_kind[6];  /* BoundaryKind of xmin, xmax, ymin, ymax, zmin, zmax */
    int face_has_p[6]; /* a pressure outlet with p= gives PRESSURE cells, without EMPTY */
    int face_order[6]; /* declaration order, -1 unspecified (no-slip); the last declared wins at edges */
    int nregions;      /* <= 16, applied in order */
    nb_region regions[16];
} nb_scene;

/* cx[j], cy[i], cz[k]: each cell's sample coordinate (its centre, or its low face for corner sampling). */
int nereus_b200_label_cells(int dim, int Nx, int Ny, int Nz, const double *cx, const double *cy, const double *cz,
                            const nb_scene *scene, uint8_t *cellTypes);

/* ---- FLIP's re-labelling from particle positions: FLIP3D::UpdateFluidCells (src/Methods/FLIP/FLIP3D.cpp:784-833)
 *      and FLIP2D::UpdateFluidCells (src/Methods/FLIP/FLIP2D.cpp:648-691), with MAC::ResetFluidCells
 *      (src/MAC.cpp:556-589). The labels come out byte for byte as the reference's serial loops leave them:
 *      every cell not SOLID, INFLOW, OUTFLOW or PRESSURE is reset to EMPTY, each particle's cell that is EMPTY
 *      becomes FLUID, then one in-place pass over the interior in (i, j, k) order fills an EMPTY cell with at least
 *      5 (3D) or 3 (2D) FLUID neighbours, a cell filled earlier in the pass counting for the later ones. ----
 * (ox, oy, oz) are the grid's FacePos(X|Y|Z, 0) (the low face of the first ring cell) and dh is SIMULATION.dh.
 * Particle p's coordinates are px[p * stride], py[p * stride], pz[p * stride] (pz unread in 2D, may be NULL): the
 * reference's own Particle array has stride 7 with px = &data[0].x, py = &data[0].y, pz = &data[0].z; separate
 * position arrays have stride 1. A particle's index along an axis is trunc((x - origin) / dh), at most N - 1, as in
 * the reference; a particle more than one cell below the grid's first face, or with a non-finite coordinate, which
 * the reference would index outside its labels with, is skipped and counted in *skipped.
 * Host form: host pointers; the call copies in and out and returns when done. skipped may be NULL. */
int nereus_b200_update_fluid_cells(int dim, int Nx, int Ny, int Nz, double ox, double oy, double oz, double dh,
                                   const double *px, const double *py, const double *pz, int64_t count,
                                   int64_t stride, uint8_t *cellTypes, int64_t *skipped);
/* Device form: cellTypes, px/py/pz, scratch and skipped (one int64, may be NULL) are DEVICE pointers on `device`;
 * the work is queued on `stream` (a cudaStream_t, NULL = the default stream) with no allocation and no host wait, so
 * it may be captured in a CUDA graph. scratch (4-byte aligned) holds the cells that the in-place pass leaves
 * undecided; nereus_b200_update_fluid_cells_scratch_bytes gives a size that always suffices (16 bytes + 4 per
 * interior cell). With less (16 bytes at least) the result is the same, and only slower when the undecided cells
 * overflow it. Calls that overlap in time on one scratch buffer race. */
size_t nereus_b200_update_fluid_cells_scratch_bytes(int dim, int Nx, int Ny, int Nz);
int nereus_b200_update_fluid_cells_device(int device, int dim, int Nx, int Ny, int Nz, double ox, double oy,
                                          double oz, double dh, const double *px, const double *py, const double *pz,
                                          int64_t count, int64_t stride, uint8_t *cellTypes, void *scratch,
                                          size_t scratch_bytes, int64_t *skipped, void *stream);

/* ---- boundary-condition replay on device fields: MAC::EnforceVelocityBC and MAC::EnforcePressureBC
 *      (src/MAC.cpp:811-865) from the lists MAC::BuildBoundaryLists makes on the host (src/MAC.cpp:613-1090), so that
 *      a stepping loop keeps u, v, w and p on the device between its sub-steps. The fields come out bit for bit as the
 *      reference's replay leaves them, ApplyOutflowFlux included. ----
 * The lists are the MAC's own, entry by entry in its order (MAC.h:450-458): solidFaceList[c]; prescribedList's
 * component and field index; copyList; ringList (kind 0 zero, 1 prescribed, 2 copy); inletFaces and outflowFaces.
 * Field indices are MAC::FieldIndex's. Components: 0 u, 1 v, 2 w. nereus_b200_bc_create copies and checks them (every
 * index inside its field, else NB_BAD_INPUT) and allocates its device memory; the enforce calls allocate nothing
 * and wait for nothing, so they may be captured in a CUDA graph. */
typedef struct nb_bc_lists
{
    int dim, Nx, Ny, Nz;                 /* ring included; Nz unread in 2D */
    const int32_t *solid[3];             /* solidFaceList[c] */
    int32_t nsolid[3];
    const int32_t *presc_comp, *presc_index; /* prescribedList */
    int32_t npresc;
    const int32_t *copy_comp, *copy_dst, *copy_src; /* copyList */
    int32_t ncopy;
    const int32_t *ring_dst, *ring_kind, *ring_src; /* ringList */
    int32_t nring;
    const int32_t *inlet_comp, *inlet_index; /* inletFaces */
    const double *inlet_area, *inlet_sign;
    int32_t ninlet;
    const int32_t *outflow_comp, *outflow_index, *outflow_outer; /* outflowFaces */
    const double *outflow_area, *outflow_sign;
    int32_t noutflow;
} nb_bc_lists;
typedef struct nb_bc nb_bc;
int nereus_b200_bc_create(int device, const nb_bc_lists *lists, nb_bc **out);
/* EnforceVelocityBC on device fields u, v, w (w unread in 2D), queued on `stream` (a cudaStream_t; NULL = the default
 * stream). presc_values: a device array of npresc doubles, entry q the boundary velocity function's component at
 * prescribedList[q]'s point and time (the caller evaluates the scene's expressions, as the reference does); NULL when
 * the scene has no boundary velocity function, which leaves the prescribed entries unwritten as the reference does. */
int nereus_b200_bc_enforce_velocity(nb_bc *bc, double *u, double *v, double *w, const double *presc_values,
                                    void *stream);
/* EnforcePressureBC on device field p. ring_values: a device array of nring doubles, read at kind-1 entries
 * (PrescribedPressure at the entry's cell and time); NULL writes 0 there, as PrescribedPressure does without a
 * pressure function. */
int nereus_b200_bc_enforce_pressure(nb_bc *bc, double *p, const double *ring_values, void *stream);
/* The number of dependency levels (launches) of each replay. */
int nereus_b200_bc_levels(const nb_bc *bc, int *velocity_levels, int *pressure_levels);
/* Host only, no device: the level each list entry is replayed in, as nereus_b200_bc_create would plan it.
 * velocity_level gets nsolid[0] + nsolid[1] + nsolid[2] + npresc + ncopy entries in that order (the reference's replay
 * order), pressure_level nring; either may be NULL. The counts of levels go to *velocity_levels, *pressure_levels. */
int nereus_b200_bc_plan(const nb_bc_lists *lists, int32_t *velocity_level, int32_t *pressure_level,
                        int *velocity_levels, int *pressure_levels);
void nereus_b200_bc_destroy(nb_bc *bc);

/* ---- batched and served solves. The reference has one solve per call from the manager thread
 *      (SimulationManager.h:345-353 -> PressureSolver3D::SolvePressure + Project); a server runs many independent
 *      pressure steps (tanks of a batch, requests of a stream) concurrently on one or more devices. Each device
 *      runs `slots_per_device` solves at once (a host thread, a solver context and a CUDA stream each; a context
 *      keeps its hierarchy while the layout bytes are unchanged, PressureLayoutChanged). A free slot takes the
 *      oldest queued request whose estimated device memory fits its device's budget: the device that frees a slot
 *      first takes the next request (least-loaded), and a finished request's slot is refilled at once. ---- */
typedef struct nb_server nb_server;

typedef struct nb_server_options
{
    int n_devices;         /* devices served (>= 1) */
    const int *devices;    /* their ordinals; NULL: 0 .. n_devices-1 */
    int slots_per_device;  /* concurrent solves per device (>= 1) */
    double hbm_budget_gb;  /* admission budget per device, GB of estimated solver memory */
    nb_options solver;     /* options of every solve; its device and stream fields are ignored */
} nb_server_options;

typedef struct nb_request
{
    int dim, Nx, Ny, Nz;            /* ring included; Nz = 1 in 2D */
    const uint8_t *cell_types;      /* copied at submission */
    const double *width[3];         /* padded Width tables (copied at submission) */
    const double *gap[3];           /* padded FaceGap tables (copied at submission) */
    int non_uniform;
    double dh;
    double *u, *v, *w, *p;          /* host fields, read when the request starts and rewritten when it completes:
                                       they must stay valid and untouched until then */
    const double *p_prev;           /* the previous pressure (incremental scheme, warm start), else NULL; read at
                                       the start */
    int scheme, needs_compat, warm_start;
    double rho, dt, tol;
    int fields_on_device;           /* 1: u, v, w, p (and p_prev) are device memory on the server's only device, their
                                       writers finished before the submission; the step runs on them in place, with
                                       no host copies */
} nb_request;

typedef struct nb_server_stats
{
    long long submitted, completed, failed, queued, running;
    double seconds;          /* since the first submission */
    double solves_per_s;     /* completed / seconds */
    double p50_ms, p99_ms;   /* submission-to-completion latency of the completed requests */
    double mean_ms;
    double admitted_gb;      /* estimated device memory of the running requests */
    long long device_completed[8]; /* completions per served device (the first 8) */
    double layout_s;         /* slots' host seconds in set_layout (hierarchy builds), summed over slots */
    double project_s;        /* slots' host seconds in the step itself (solve, projection, copies), summed */
} nb_server_stats;

void nereus_b200_default_server_options(nb_server_options *o);
int nereus_b200_server_create(nb_server **srv, const nb_server_options *opt);
/* Waits for the requests in flight to finish; queued requests that have not started are dropped. */
void nereus_b200_server_destroy(nb_server *srv);
/* Queues one request; *ticket identifies it. NB_BAD_INPUT: malformed, or larger than a device's budget. */
int nereus_b200_submit(nb_server *srv, const nb_request *req, uint64_t *ticket);
/* NB_BUSY while queued or running; then the request's nb_status, with *out its report. */
int nereus_b200_poll(nb_server *srv, uint64_t ticket, nb_result *out);
/* As poll, blocking up to timeout_s seconds (< 0: no limit) for completion. */
int nereus_b200_wait(nb_server *srv, uint64_t ticket, double timeout_s, nb_result *out);
int nereus_b200_server_stats(nb_server *srv, nb_server_stats *stats);
/* Starts the statistics afresh (counts, latencies, the clock) from now; queued and running requests are kept. */
int nereus_b200_server_reset_stats(nb_server *srv);
/* Estimated device bytes of one solve (the admission cost): fields, right-hand side and solution, level vectors. */
double nereus_b200_request_bytes(int dim, int Nx, int Ny, int Nz, int precision);
/* Host only: a deterministic least-loaded assignment of n requests with the given costs to k devices (or processes):
 * in submission order, each goes to the device with the smallest assigned total (lowest index on ties). */
int nereus_b200_plan(const double *costs, int n, int k, int *device_of);

/* ---- batched solves: one pressure step for each of many grids of the same shape, advanced together. Replaces, for
 *      a caller with many independent systems (FLIP tanks, ensemble members), one SolvePressureSystem call per
 *      system (PressureSettings.h:578-624), each of which waits for its solver alone. Every kernel of a CG iteration
 *      is one launch over all requests still iterating (a device-side work list of requests, compacted after each
 *      iteration as requests converge), the iteration runs as a captured CUDA graph with a WHILE node, and each
 *      request keeps its own labels, multigrid hierarchy, vectors, reductions, tolerance and iteration count. A
 *      request's result does not depend on the rest of the batch (alone or in any mix, the same bits); it agrees
 *      with nereus_b200_project_device on the same request within the solve's tolerance.
 *      Mixed precision; uniform 3D grids whose multigrid levels above the coarse end have Nz even. ---- */
typedef struct nb_batch nb_batch;

typedef struct nb_batch_item
{
    double *u, *v, *w, *p; /* device fields of the request's slot (as nereus_b200_project_device) */
    double rho, dt;
    int needs_compat;
    double tol;
} nb_batch_item;

#define NB_BATCH_MAX_LEVELS 16
typedef struct nb_batch_info
{
    int capacity, levels, tail_start;
    long long loop_launches;                   /* kernels one batched CG iteration launches */
    double tune_ms;                            /* device time the autotuner spent */
    int march[NB_BATCH_MAX_LEVELS][5];         /* per split level: the march length of the first sweep, a half-sweep,
                                                  the residual, the restriction, the prolongation */
    int restrict_mode[NB_BATCH_MAX_LEVELS];    /* 1: one thread per coarse cell; 2: one per four */
} nb_batch_info;

/* capacity: the most requests one call takes (1 .. 1024); opt->precision must be NB_PRECISION_MIXED */
int nereus_b200_batch_create(nb_batch **batch, const nb_options *opt, int capacity);
void nereus_b200_batch_destroy(nb_batch *batch);
/* the layout of slot `slot` (as nereus_b200_set_layout; unchanged bytes keep its hierarchy) */
int nereus_b200_batch_set_layout(nb_batch *batch, int slot, int dim, int Nx, int Ny, int Nz, const uint8_t *cellTypes,
                                 const double *const width[3], const double *const gap[3], int nonUniform, double dh);
/* The Chorin step of slots 0 .. count-1 with items[i]'s device fields; results[i] gets each one's report. Returns the
 * worst status. NB_BAD_INPUT when the slots' shapes differ or do not take the batched form. */
int nereus_b200_batch_project_device(nb_batch *batch, int count, const nb_batch_item *items, nb_result *results);
int nereus_b200_batch_info(nb_batch *batch, nb_batch_info *info);
/* The autotuner (host only). choose: the candidate index to keep given the candidates' times (the fastest, unless
 * the fallback is within 3% of it; ties within 0.5% to the earlier one). key: the cache key of a (grid, level,
 * kernel kind 0-4, capacity) into buf, returning its length. The cache holds one line per key, "key|S|mode|us"
 * (mode records a restriction level's kernel; it is not tuned and a loaded mode is not applied, only S is):
 * dump writes it into buf (returning its full length), load adds lines of that form (returning the count, or
 * NB_BAD_INPUT for a malformed text), clear empties it. */
int nereus_b200_tune_choose(int n, const double *times, int fallback);
/* The x groups a stretched 3D level's coarsening makes (x_groups = 1; host only): n interior x widths, yz_min the
 * thinnest interior y or z width. Left to right, two cells form one coarse cell when together they are at most
 * 1.5 coarse y/z cells (3 yz_min) wide, else a cell stays whole. Writes each group's cell count (1 or 2) into
 * counts (room for n) and returns the number of groups, or NB_BAD_INPUT. */
int nereus_b200_x_groups(const double *widths, int n, double yz_min, int32_t *counts);
/* The same groups as the transfer maps the kernels read (host only): xp[j] for the fine x index j = 0 .. n+1 (rings
 * included): parent (bits 0-14), other contributor (bits 15-29), bit 30 when the parent has one child; xr[J] for the
 * coarse x index J: first child (bits 0-14), bit 15 two children, bit 16 / 17 the group before / after has two.
 * Returns the coarse extent Nc (rings included; xr needs room for n + 2), 0 when the groups are the regular pairing
 * of every axis (nothing written), or NB_BAD_INPUT. */
int nereus_b200_x_maps(const double *widths, int n, double yz_min, int32_t *xp, int32_t *xr);
int nereus_b200_tune_key(int Nx, int Ny, int Nz, int level, int kind, int capacity, char *buf, int size);
int nereus_b200_tune_cache_dump(char *buf, int size);
int nereus_b200_tune_cache_load(const char *text);
void nereus_b200_tune_cache_clear(void);

/* ---- IDP numbering without allocation. No counterpart in the reference. It gives the same numbering as
 *      nereus_b200_get_idp after nereus_b200_set_layout, for callers that must not allocate device memory at the
 *      point they renumber. ----
 * cellTypes (Nx*Ny*Nz bytes), idp (Nx*Ny*Nz int32) and n (one int32) are DEVICE pointers on `device`; the call is
 * asynchronous on `stream` (a cudaStream_t, NULL = the default stream). idp gets -1 off the system, *n the count.
 * Makes no cudaMalloc/cudaFree: its scratch is one fixed 2 MiB array per device, enough for grids of at most
 * NB_NOALLOC_MAX_LINES interior lines ((Ny-2)*(Nx-2) in 3D, Ny-2 in 2D); larger grids get NB_BAD_INPUT.
 * The first call on a device looks up that array's address (and may load the library's device code), so make it
 * before any stream capture begins; after a cudaDeviceReset the next call looks it up again, so make that one
 * before any capture too. Calls that overlap in time on one device share the scratch and race. */
#define NB_NOALLOC_MAX_LINES 262144
int nereus_b200_number_unknowns_noalloc(int device, int dim, int Nx, int Ny, int Nz, const uint8_t *cellTypes,
                                        int32_t *idp, int32_t *n, void *stream);

#ifdef __cplusplus
}
#endif
#endif
