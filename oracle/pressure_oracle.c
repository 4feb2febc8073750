/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the NEREUS pressure projection (RaphaelLaroca/NEREUS_CFD): tests/ check the B200 path's
 * results against it, and bench.py's CPU-baseline leg times it. The product library never links, loads or calls this
 * file.
 *
 * Parity pin: tests/test_oracle_golden.py checks every function here against the reference's own outputs
 * (the .npz fixtures under tests/golden, written by tests/golden/make_golden.py from oracle/_ref/ref_harness, which is compiled from
 * the reference sources) -- cell types, IDP numbering and the CSR matrix bit-exact, b bit-exact, x to the CG
 * tolerance -- and against the reference's known-answer tests (tests/suite_pressure.cpp:55-57,166-169,230:
 * a linear Dirichlet field is reproduced exactly).
 *
 * Layout (src/headers/Core/MAC.h:235-254, 369-374): cell (i,j,k) = (y,x,z) at (i*Nx + j)*Nz + k; u has Nx+1 along x,
 * v has Ny+1 along y, w has Nz+1 along z. A 2D grid is the 3D layout with Nz = 1 and no z faces. Nx, Ny, Nz include
 * the one-cell border ring. Spacing tables are the reference's padded ones (MAC.h:439-448, src/MAC.cpp:165-175,
 * 519-525): width[a][n+1] = Width(a, n) for n = -1..N, gap[a][n+1] = FaceGap(a, n) for n = -1..N-1.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Cell types, src/headers/Core/Definitions.h:191-196. */
enum { FLUID = 0, SOLID = 1, EMPTY = 2, INFLOW = 3, PRESSURE = 4, OUTFLOW = 5 };
/* Boundary kinds, Definitions.h:212. */
enum { BC_NOSLIP = 0, BC_SLIP, BC_MOVING, BC_INLET, BC_PRESSURE_OUTLET, BC_OUTFLOW };
/* Scene primitives and regions (src/headers/Core/Scene.h). */
enum { PRIM_BOX = 0, PRIM_SPHERE = 1, PRIM_CYLINDER = 2, PRIM_PLANE = 3 };
enum { REGION_SOLID = 0, REGION_FLUID = 1, REGION_EMPTY = 2 };

typedef struct
{
    int dim, Nx, Ny, Nz; /* Nz = 1 in 2D */
    int nonuniform;
    double dh;
    const double *width[3]; /* padded, N + 2 entries */
    const double *gap[3];   /* padded, N + 1 entries */
    const uint8_t *types;
} or_grid;

typedef struct
{
    int kind, region, axis, invert;
    double p0[3], p1[3], radius;
} or_region;

typedef struct
{
    int face_kind[6];  /* BoundaryKind per face: xmin, xmax, ymin, ymax, zmin, zmax */
    int face_has_p[6]; /* a pressure outlet with p= is a PRESSURE cell, without one EMPTY */
    int face_order[6]; /* declaration order; -1 for an unspecified face (no-slip) */
    int nregions;
    or_region regions[16];
} or_scene;

static inline double Wd(const or_grid *g, int a, int n) { return g->width[a][n + 1]; }
static inline double Gp(const or_grid *g, int a, int n) { return g->gap[a][n + 1]; }
static inline size_t Cell(const or_grid *g, int i, int j, int k) { return ((size_t)i * g->Nx + j) * g->Nz + k; }
static inline int T(const or_grid *g, int i, int j, int k) { return g->types[Cell(g, i, j, k)]; }
static inline int IsDirichlet(int t) { return t == EMPTY || t == PRESSURE; }
static inline size_t IU(const or_grid *g, int i, int j, int k) { return ((size_t)i * (g->Nx + 1) + j) * g->Nz + k; }
static inline size_t IV(const or_grid *g, int i, int j, int k) { return ((size_t)i * g->Nx + j) * g->Nz + k; }
static inline size_t IW(const or_grid *g, int i, int j, int k) { return ((size_t)i * g->Nx + j) * (g->Nz + 1) + k; }

/* ---- a1: cell types from the scene (Scene.h:265-300 Distance, :352-366 Contains, :566-575 WinningFace,
 *          :613-621 FacesAtCell, :639-673 CellTypeAt, :677-686 CellTypeOf) ---- */
static double PrimDistance(const or_region *p, int dim, double x, double y, double z)
{
    const int axes = dim == 2 ? 2 : 3;
    double d = 0.0;
    if (p->kind == PRIM_BOX)
    {
        const double c[3] = {x, y, z};
        double outside = 0.0, inside = -1e30;
        for (int a = 0; a < axes; a++)
        {
            const double dlo = p->p0[a] - c[a];
            const double dhi = c[a] - p->p1[a];
            const double dm = dlo > dhi ? dlo : dhi;
            if (dm > 0.0) outside += dm * dm;
            inside = inside > dm ? inside : dm;
        }
        d = outside > 0.0 ? sqrt(outside) : inside;
    }
    else if (p->kind == PRIM_SPHERE)
    {
        const double dx = x - p->p0[0], dy = y - p->p0[1];
        const double dz = axes == 3 ? (z - p->p0[2]) : 0.0;
        d = sqrt(dx * dx + dy * dy + dz * dz) - p->radius;
    }
    else if (p->kind == PRIM_CYLINDER)
    {
        double a1, a2;
        if (p->axis == 0) { a1 = y - p->p0[1]; a2 = z - p->p0[2]; }
        else if (p->axis == 1) { a1 = x - p->p0[0]; a2 = z - p->p0[2]; }
        else { a1 = x - p->p0[0]; a2 = y - p->p0[1]; }
        d = sqrt(a1 * a1 + a2 * a2) - p->radius;
    }
    else
    {
        const double nx = p->p1[0], ny = p->p1[1];
        const double nz = axes == 3 ? p->p1[2] : 0.0;
        const double len = sqrt(nx * nx + ny * ny + nz * nz);
        const double inv = len > 0.0 ? 1.0 / len : 0.0;
        const double dzc = axes == 3 ? (z - p->p0[2]) : 0.0;
        d = ((x - p->p0[0]) * nx + (y - p->p0[1]) * ny + dzc * nz) * inv;
    }
    return p->invert ? -d : d;
}

static int CellTypeOfFace(const or_scene *s, int f)
{
    switch (s->face_kind[f])
    {
    case BC_INLET: return INFLOW;
    case BC_OUTFLOW: return OUTFLOW;
    case BC_PRESSURE_OUTLET: return s->face_has_p[f] ? PRESSURE : EMPTY;
    default: return SOLID;
    }
}

/* cx[j], cy[i], cz[k]: the sample coordinate of each cell (the centre, or the cell's low face for corner sampling),
 * as Scene::AxisCoord reads them from SIMULATION.spacing. */
int or_label_cells(int dim, int Nx, int Ny, int Nz, const double *cx, const double *cy, const double *cz,
                   const or_scene *s, uint8_t *types)
{
    const int nz = dim == 3 ? Nz : 1;
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++)
            for (int k = 0; k < nz; k++)
            {
                const double x = cx[j], y = cy[i], z = dim == 3 ? cz[k] : cz[0];
                int type = FLUID;
                for (int r = 0; r < s->nregions; r++)
                {
                    const or_region *p = &s->regions[r];
                    if (!(PrimDistance(p, dim, x, y, z) < 0.0)) continue;
                    type = p->region == REGION_SOLID ? SOLID : (p->region == REGION_FLUID ? FLUID : EMPTY);
                }
                const int on[6] = {j == 0, j == Nx - 1, i == 0, i == Ny - 1, k == 0, k == Nz - 1};
                int best = -1, bestOrder = -2;
                for (int f = 0; f < 6; f++)
                {
                    if (!on[f] || (dim == 2 && f >= 4)) continue;
                    if (s->face_order[f] > bestOrder) { bestOrder = s->face_order[f]; best = f; }
                }
                if (best >= 0) type = CellTypeOfFace(s, best);
                types[((size_t)i * Nx + j) * nz + k] = (uint8_t)type;
            }
    return 0;
}

/* ---- a2: face coefficients, ring factors, assembly ---- */

/* Face coefficients toward (i+1, i-1, j+1, j-1, k+1, k-1): PressureSolver3D.cpp:47-63 (3D), the c[] table of
 * PressureSolver2D.cpp:123-126 (2D). */
static void FaceCoefs(const or_grid *g, int i, int j, int k, double c[6])
{
    if (g->dim == 2)
    {
        c[0] = Wd(g, 0, j) / Gp(g, 1, i);
        c[1] = Wd(g, 0, j) / Gp(g, 1, i - 1);
        c[2] = Wd(g, 1, i) / Gp(g, 0, j);
        c[3] = Wd(g, 1, i) / Gp(g, 0, j - 1);
        c[4] = c[5] = 0.0;
        return;
    }
    if (!g->nonuniform)
    {
        for (int q = 0; q < 6; q++) c[q] = 1.0;
        return;
    }
    const double ax = Wd(g, 1, i) * Wd(g, 2, k); /* FaceArea, MAC.h:91-92 */
    const double ay = Wd(g, 0, j) * Wd(g, 2, k);
    const double az = Wd(g, 0, j) * Wd(g, 1, i);
    c[0] = ay / Gp(g, 1, i);
    c[1] = ay / Gp(g, 1, i - 1);
    c[2] = ax / Gp(g, 0, j);
    c[3] = ax / Gp(g, 0, j - 1);
    c[4] = az / Gp(g, 2, k);
    c[5] = az / Gp(g, 2, k - 1);
}

static const int DI[6] = {1, -1, 0, 0, 0, 0};
static const int DJ[6] = {0, 0, 1, -1, 0, 0};
static const int DK[6] = {0, 0, 0, 0, 1, -1};

/* DirichletRingFactor, PressureSettings.h:307-310. */
static inline double DirichletRingFactor(const or_grid *g, int a, int n, int s)
{
    return Gp(g, a, s < 0 ? n - 1 : n) / (0.5 * Wd(g, a, n));
}

/* RingFactor3D, PressureSolver3D.cpp:80-87; RingFactor2D, PressureSolver2D.cpp:55-60. */
static double RingFactor(const or_grid *g, int i, int j, int k, int q)
{
    const int ni = i + DI[q], nj = j + DJ[q], nk = k + DK[q];
    if (!IsDirichlet(T(g, ni, nj, nk))) return 1.0;
    const int onRing = ni == 0 || ni == g->Ny - 1 || nj == 0 || nj == g->Nx - 1 ||
                       (g->dim == 3 && (nk == 0 || nk == g->Nz - 1));
    if (!onRing) return 1.0;
    const int s = (q % 2 == 0) ? 1 : -1;
    return q < 2 ? DirichletRingFactor(g, 1, i, s) : (q < 4 ? DirichletRingFactor(g, 0, j, s) : DirichletRingFactor(g, 2, k, s));
}

static inline double MatrixScale(const or_grid *g) { return g->nonuniform ? 1.0 : 1.0 / (g->dh * g->dh); }

static inline int KLo(const or_grid *g) { return g->dim == 3 ? 1 : 0; }
static inline int KHi(const or_grid *g) { return g->dim == 3 ? g->Nz - 1 : 1; }
static inline int NQ(const or_grid *g) { return g->dim == 3 ? 6 : 4; }

/* IDP numbering, PressureSolver3D.cpp:133-139 / PressureSolver2D.cpp:104-109. Returns n. */
int or_number_unknowns(const or_grid *g, int32_t *idp)
{
    const size_t cells = (size_t)g->Nx * g->Ny * g->Nz;
    for (size_t c = 0; c < cells; c++) idp[c] = -1;
    int n = 0;
    for (int i = 1; i < g->Ny - 1; i++)
        for (int j = 1; j < g->Nx - 1; j++)
            for (int k = KLo(g); k < KHi(g); k++)
                if (T(g, i, j, k) == FLUID) idp[Cell(g, i, j, k)] = n++;
    return n;
}

/* The assembled matrix, AssembleSystem (PressureSolver3D.cpp:128-178, PressureSolver2D.cpp:100-152), written as
 * the CSR that Eigen's setFromTriplets + makeCompressed leaves: rows in IDP order, columns ascending, the diagonal
 * only when non-zero. rowptr has n+1 entries; col/val need at most 7n (3D) / 5n (2D). Returns nnz; *singular is
 * set when no row touches a Dirichlet neighbour. */
int or_assemble(const or_grid *g, const int32_t *idp, int32_t *rowptr, int32_t *col, double *val, int *singular)
{
    const double scale = MatrixScale(g);
    int nnz = 0, row = 0, dirichlet = 0;
    const int nq = NQ(g);
    for (int i = 1; i < g->Ny - 1; i++)
        for (int j = 1; j < g->Nx - 1; j++)
            for (int k = KLo(g); k < KHi(g); k++)
            {
                const int r = idp[Cell(g, i, j, k)];
                if (r < 0) continue;
                double c[6];
                FaceCoefs(g, i, j, k, c);
                int ecol[7];
                double eval[7];
                int ne = 0;
                double diag = 0.0;
                for (int q = 0; q < nq; q++)
                    if (T(g, i + DI[q], j + DJ[q], k + DK[q]) == FLUID)
                    {
                        diag -= c[q];
                        const int cl = idp[Cell(g, i + DI[q], j + DJ[q], k + DK[q])];
                        if (cl >= 0) { ecol[ne] = cl; eval[ne] = scale * c[q]; ne++; }
                        else dirichlet = 1;
                    }
                for (int q = 0; q < nq; q++)
                    if (IsDirichlet(T(g, i + DI[q], j + DJ[q], k + DK[q])))
                    {
                        diag -= c[q] * RingFactor(g, i, j, k, q);
                        dirichlet = 1;
                    }
                if (diag != 0.0) { ecol[ne] = r; eval[ne] = scale * diag; ne++; }
                /* ascending columns (insertion sort of at most 7) */
                for (int a = 1; a < ne; a++)
                    for (int b = a; b > 0 && ecol[b - 1] > ecol[b]; b--)
                    {
                        const int tc = ecol[b]; ecol[b] = ecol[b - 1]; ecol[b - 1] = tc;
                        const double tv = eval[b]; eval[b] = eval[b - 1]; eval[b - 1] = tv;
                    }
                rowptr[row] = nnz;
                for (int e = 0; e < ne; e++) { col[nnz] = ecol[e]; val[nnz] = eval[e]; nnz++; }
                row++;
                (void)r;
            }
    rowptr[row] = nnz;
    *singular = !dirichlet;
    return nnz;
}

/* ---- a3: divergence and right-hand side ---- */

/* MAC::GetDivergencyAt, src/MAC.cpp:349-367 (3D), :443-456 (2D). */
double or_divergence_at(const or_grid *g, const double *u, const double *v, const double *w, int i, int j, int k)
{
    if (T(g, i, j, k) != FLUID) return 0.0;
    if (g->dim == 2)
    {
        if (g->nonuniform)
        {
            const double dx = Wd(g, 0, j), dy = Wd(g, 1, i);
            const double fluxU = (u[IU(g, i, j + 1, 0)] - u[IU(g, i, j, 0)]) * dy;
            const double fluxV = (v[IV(g, i + 1, j, 0)] - v[IV(g, i, j, 0)]) * dx;
            return (fluxU + fluxV) / (dx * dy);
        }
        const double divU = (u[IU(g, i, j + 1, 0)] - u[IU(g, i, j, 0)]) / g->dh;
        const double divV = (v[IV(g, i + 1, j, 0)] - v[IV(g, i, j, 0)]) / g->dh;
        return divU + divV;
    }
    if (g->nonuniform)
    {
        const double dx = Wd(g, 0, j), dy = Wd(g, 1, i), dz = Wd(g, 2, k);
        const double fluxU = (u[IU(g, i, j + 1, k)] - u[IU(g, i, j, k)]) * dy * dz;
        const double fluxV = (v[IV(g, i + 1, j, k)] - v[IV(g, i, j, k)]) * dx * dz;
        const double fluxW = (w[IW(g, i, j, k + 1)] - w[IW(g, i, j, k)]) * dx * dy;
        return (fluxU + fluxV + fluxW) / (dx * dy * dz);
    }
    const double divU = (u[IU(g, i, j + 1, k)] - u[IU(g, i, j, k)]) / g->dh;
    const double divV = (v[IV(g, i + 1, j, k)] - v[IV(g, i, j, k)]) / g->dh;
    const double divW = (w[IW(g, i, j, k + 1)] - w[IW(g, i, j, k)]) / g->dh;
    return divU + divV + divW;
}

/* DirichletSum (Chorin), PressureSolver3D.cpp:248-260 / PressureSolver2D.cpp:223-235. */
static double DirichletSum(const or_grid *g, const double *p, int i, int j, int k)
{
    double c[6];
    FaceCoefs(g, i, j, k, c);
    double s = 0.0;
    for (int q = 0; q < NQ(g); q++)
        if (T(g, i + DI[q], j + DJ[q], k + DK[q]) == PRESSURE)
            s += c[q] * RingFactor(g, i, j, k, q) * p[Cell(g, i + DI[q], j + DJ[q], k + DK[q])];
    return s;
}

/* The right-hand side before the compatibility step, SolveScheme's loop (PressureSolver3D.cpp:288-298,
 * PressureSolver2D.cpp:263-272): b = rho/dt * div * V - scale * DirichletSum. */
void or_rhs(const or_grid *g, const int32_t *idp, const double *u, const double *v, const double *w,
            const double *p, double rho, double dt, double *b)
{
    const double scale = MatrixScale(g);
    const double rhoDt = rho / dt;
    for (int i = 1; i < g->Ny - 1; i++)
        for (int j = 1; j < g->Nx - 1; j++)
            for (int k = KLo(g); k < KHi(g); k++)
            {
                const int id = idp[Cell(g, i, j, k)];
                if (id < 0) continue;
                double vol = 1.0;
                if (g->nonuniform)
                    vol = g->dim == 3 ? Wd(g, 0, j) * Wd(g, 1, i) * Wd(g, 2, k) : Wd(g, 0, j) * Wd(g, 1, i);
                b[id] = rhoDt * or_divergence_at(g, u, v, w, i, j, k) * vol - scale * DirichletSum(g, p, i, j, k);
            }
}

/* ---- a4: compatibility, PressureSolver3D.cpp:300-307 + SubtractMean (PressureSettings.h:314-321) ---- */
void or_compat(double *b, int n)
{
    for (int pass = 0; pass < 2; pass++)
    {
        double m = 0.0;
        for (int q = 0; q < n; q++) m += b[q];
        m /= (double)n;
        for (int q = 0; q < n; q++) b[q] -= m;
    }
}

/* ---- a5: the solve. Eigen 3.3.7 ConjugateGradient with DiagonalPreconditioner, as the reference's CPU path runs
 * it (PressureSettings.h:386-396, 400, 453): include/eigen-3.3.7/Eigen/src/IterativeLinearSolvers/
 * ConjugateGradient.h:26-89 and BasicPreconditioners.h:64-92. Stops at ||r||^2 < max(tol^2 ||b||^2, DBL_MIN).
 * Returns the iterations; *err = ||r||/||b||. ---- */
static void Spmv(const int32_t *rp, const int32_t *cl, const double *val, int n, const double *x, double *y)
{
    for (int r = 0; r < n; r++)
    {
        double s = 0.0;
        for (int e = rp[r]; e < rp[r + 1]; e++) s += val[e] * x[cl[e]];
        y[r] = s;
    }
}
static double Dot(const double *a, const double *b, int n)
{
    double s = 0.0;
    for (int q = 0; q < n; q++) s += a[q] * b[q];
    return s;
}

int or_cg(const int32_t *rp, const int32_t *cl, const double *val, int n, const double *b, double *x, double tol,
          int maxIters, double *err)
{
    double *inv = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double *r = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double *p = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double *z = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double *t = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    for (int q = 0; q < n; q++)
    {
        inv[q] = 1.0;
        for (int e = rp[q]; e < rp[q + 1]; e++)
            if (cl[e] == q && val[e] != 0.0) inv[q] = 1.0 / val[e];
    }
    int it = 0;
    Spmv(rp, cl, val, n, x, t);
    for (int q = 0; q < n; q++) r[q] = b[q] - t[q];
    const double rhs2 = Dot(b, b, n);
    if (rhs2 == 0.0)
    {
        for (int q = 0; q < n; q++) x[q] = 0.0;
        *err = 0.0;
        goto done;
    }
    {
        const double thr = fmax(tol * tol * rhs2, 2.2250738585072014e-308);
        double rn2 = Dot(r, r, n);
        if (rn2 < thr) { *err = sqrt(rn2 / rhs2); goto done; }
        for (int q = 0; q < n; q++) p[q] = inv[q] * r[q];
        double absNew = Dot(r, p, n);
        while (it < maxIters)
        {
            Spmv(rp, cl, val, n, p, t);
            const double alpha = absNew / Dot(p, t, n);
            for (int q = 0; q < n; q++) x[q] += alpha * p[q];
            for (int q = 0; q < n; q++) r[q] -= alpha * t[q];
            rn2 = Dot(r, r, n);
            if (rn2 < thr) break;
            for (int q = 0; q < n; q++) z[q] = inv[q] * r[q];
            const double absOld = absNew;
            absNew = Dot(r, z, n);
            const double beta = absNew / absOld;
            for (int q = 0; q < n; q++) p[q] = z[q] + beta * p[q];
            it++;
        }
        *err = sqrt(rn2 / rhs2);
    }
done:
    free(inv); free(r); free(p); free(z); free(t);
    return it;
}

/* ---- a6: LevelPressure's mean removal (PressureSolver3D.cpp:181-187): p -= mean(p) for a singular system with
 * the compatibility condition on. The inflow p= shift that follows needs the scene's expressions; it is
 * or_level_shift below, given the level values. ---- */
void or_level_mean(double *x, int n)
{
    if (n <= 0) return;
    double m = 0.0;
    for (int q = 0; q < n; q++) m += x[q];
    m /= (double)n;
    for (int q = 0; q < n; q++) x[q] -= m;
}

/* AccumulateLevel3D's sum (PressureSolver3D.cpp:15-30,188-211): for each (level, p1, p2, sR, s1, s2) record the
 * shift level - (p1 + (p1 - p2)(sR - s1)/(s1 - s2)); x += mean shift. rec has 6 doubles per entry, p1/p2 given as
 * unknown indices in rec_ids (2 per entry). */
void or_level_shift(double *x, int n, const double *rec, const int32_t *rec_ids, int nrec)
{
    if (nrec <= 0 || n <= 0) return;
    double sum = 0.0;
    for (int e = 0; e < nrec; e++)
    {
        const double level = rec[6 * e], sR = rec[6 * e + 3], s1 = rec[6 * e + 4], s2 = rec[6 * e + 5];
        const double p1 = x[rec_ids[2 * e]], p2 = x[rec_ids[2 * e + 1]];
        sum += level - (p1 + (p1 - p2) * (sR - s1) / (s1 - s2));
    }
    for (int q = 0; q < n; q++) x[q] += sum / nrec;
}

/* ---- a7: scatter and the pressure ring (PressureSolver3D.cpp:321-328; MAC::EnforcePressureBC src/MAC.cpp:866-871
 * replaying BuildRingList src/MAC.cpp:1064-1096 and RecordRing MAC.h:482-487): EMPTY ring cells 0, PRESSURE ring
 * cells keep the prescribed value already in p, any other ring cell copies the cell one step inward, y faces
 * first, then x, then z. ---- */
void or_scatter(const or_grid *g, const int32_t *idp, const double *x, double *p)
{
    const size_t cells = (size_t)g->Nx * g->Ny * g->Nz;
    for (size_t c = 0; c < cells; c++)
        if (idp[c] >= 0) p[c] = x[idp[c]];
}

static inline void RingEntry(const or_grid *g, double *p, int i, int j, int k, int si, int sj, int sk)
{
    const int t = T(g, i, j, k);
    const size_t d = Cell(g, i, j, k);
    if (t == EMPTY) p[d] = 0.0;
    else if (t == PRESSURE) { /* prescribed: the caller's value stands */ }
    else p[d] = p[Cell(g, si, sj, sk)];
}

void or_ring_replay(const or_grid *g, double *p)
{
    const int Nx = g->Nx, Ny = g->Ny, Nz = g->Nz;
    if (g->dim == 2)
    {
        for (int j = 0; j < Nx; j++) { RingEntry(g, p, 0, j, 0, 1, j, 0); RingEntry(g, p, Ny - 1, j, 0, Ny - 2, j, 0); }
        for (int i = 0; i < Ny; i++) { RingEntry(g, p, i, 0, 0, i, 1, 0); RingEntry(g, p, i, Nx - 1, 0, i, Nx - 2, 0); }
        return;
    }
    for (int j = 0; j < Nx; j++)
        for (int k = 0; k < Nz; k++) { RingEntry(g, p, 0, j, k, 1, j, k); RingEntry(g, p, Ny - 1, j, k, Ny - 2, j, k); }
    for (int i = 0; i < Ny; i++)
        for (int k = 0; k < Nz; k++) { RingEntry(g, p, i, 0, k, i, 1, k); RingEntry(g, p, i, Nx - 1, k, i, Nx - 2, k); }
    for (int i = 0; i < Ny; i++)
        for (int j = 0; j < Nx; j++) { RingEntry(g, p, i, j, 0, i, j, 1); RingEntry(g, p, i, j, Nz - 1, i, j, Nz - 2); }
}

/* ---- a8: the projection, ProjectPressure (PressureSolver3D.cpp:417-438, PressureSolver2D.cpp:382-395) with
 * ProjectionGradient (PressureSolver3D.cpp:405-414, PressureSolver2D.cpp:370-379), MAC::GetGradP (MAC.h:149-154,
 * 363-367) and FaceGate (MAC.h:271-274, 394-397, 502-507): u -= dt/rho grad p on every face with no solid side. ---- */
static double ProjGrad(const or_grid *g, int a, int i, int j, int k, const double *p)
{
    double grad;
    if (a == 0) grad = (p[Cell(g, i, j, k)] - p[Cell(g, i, j - 1, k)]) / Gp(g, 0, j - 1);
    else if (a == 1) grad = (p[Cell(g, i, j, k)] - p[Cell(g, i - 1, j, k)]) / Gp(g, 1, i - 1);
    else grad = (p[Cell(g, i, j, k)] - p[Cell(g, i, j, k - 1)]) / Gp(g, 2, k - 1);
    const int n = a == 0 ? j : (a == 1 ? i : k);
    const int N = a == 0 ? g->Nx : (a == 1 ? g->Ny : g->Nz);
    if (n != 1 && n != N - 1) return grad;
    if (g->dim == 2)
    {
        /* PressureSolver2D.cpp:370-379 tests n == 1 first, then n == N-1. */
        if (n == 1 && IsDirichlet(a == 0 ? T(g, i, 0, 0) : T(g, 0, j, 0))) return grad * DirichletRingFactor(g, a, 1, -1);
        if (n == N - 1 && IsDirichlet(a == 0 ? T(g, i, N - 1, 0) : T(g, N - 1, j, 0)))
            return grad * DirichletRingFactor(g, a, N - 2, +1);
        return grad;
    }
    const int r = n == 1 ? 0 : N - 1;
    const int t = a == 0 ? T(g, i, r, k) : (a == 1 ? T(g, r, j, k) : T(g, i, j, r));
    if (!IsDirichlet(t)) return grad;
    return n == 1 ? grad * DirichletRingFactor(g, a, 1, -1) : grad * DirichletRingFactor(g, a, N - 2, +1);
}

static inline int Wall(int a, int b) { return a == SOLID || b == SOLID; }

void or_project(const or_grid *g, double *u, double *v, double *w, const double *p, double rho, double dt)
{
    const int nx = g->Nx, ny = g->Ny, nz = g->Nz;
    const double f = dt / rho;
    const int k0 = KLo(g), k1 = KHi(g);
    for (int i = 1; i < ny - 1; i++)
        for (int j = 1; j < nx; j++)
            for (int k = k0; k < k1; k++)
                if (!Wall(T(g, i, j, k), T(g, i, j - 1, k))) u[IU(g, i, j, k)] = u[IU(g, i, j, k)] - f * ProjGrad(g, 0, i, j, k, p);
    for (int i = 1; i < ny; i++)
        for (int j = 1; j < nx - 1; j++)
            for (int k = k0; k < k1; k++)
                if (!Wall(T(g, i, j, k), T(g, i - 1, j, k))) v[IV(g, i, j, k)] = v[IV(g, i, j, k)] - f * ProjGrad(g, 1, i, j, k, p);
    if (g->dim == 2) return;
    for (int i = 1; i < ny - 1; i++)
        for (int j = 1; j < nx - 1; j++)
            for (int k = 1; k < nz; k++)
                if (!Wall(T(g, i, j, k), T(g, i, j, k - 1))) w[IW(g, i, j, k)] = w[IW(g, i, j, k)] - f * ProjGrad(g, 2, i, j, k, p);
}

/* Max |GetDivergencyAt| over the grid (0 at every non-FLUID cell). */
double or_max_divergence(const or_grid *g, const double *u, const double *v, const double *w)
{
    double m = 0.0;
    for (int i = 1; i < g->Ny - 1; i++)
        for (int j = 1; j < g->Nx - 1; j++)
            for (int k = KLo(g); k < KHi(g); k++)
            {
                const double d = fabs(or_divergence_at(g, u, v, w, i, j, k));
                if (d > m) m = d;
            }
    return m;
}

/* ||b - A x||_2 with the CSR matrix. */
double or_residual_norm(const int32_t *rp, const int32_t *cl, const double *val, int n, const double *b, const double *x)
{
    double s = 0.0;
    for (int r = 0; r < n; r++)
    {
        double ax = 0.0;
        for (int e = rp[r]; e < rp[r + 1]; e++) ax += val[e] * x[cl[e]];
        const double d = b[r] - ax;
        s += d * d;
    }
    return sqrt(s);
}

/* One particle coordinate to a cell index along an axis with N cells, as UpdateFluidCells does it
 * (src/Methods/FLIP/FLIP3D.cpp:796-802): truncation toward zero of (x - origin) / dh, clamped above to N - 1. The
 * reference has no lower clamp: an index below 0 (x more than one cell below the grid's first face) or a non-finite
 * coordinate reads outside the labels there. Here such a particle is skipped (-1), and so is it in the B200 kernel.
 * A quotient at or beyond N (including +inf) takes N - 1 without converting it. */
static inline int ParticleIndex(double x, double origin, double dh, int N)
{
    const double q = (x - origin) / dh;
    if (!(q > -1.0)) return -1;
    if (q >= (double)N) return N - 1;
    return (int)q;
}

/* FLIP3D::UpdateFluidCells (src/Methods/FLIP/FLIP3D.cpp:784-833) and FLIP2D::UpdateFluidCells
 * (src/Methods/FLIP/FLIP2D.cpp:648-691), in their order:
 *   1. MAC::ResetFluidCells (src/MAC.cpp:556-589): every cell that is not SOLID, INFLOW, OUTFLOW or PRESSURE becomes
 *      EMPTY, ring included;
 *   2. each particle's cell, if EMPTY, becomes FLUID;
 *   3. one pass over the interior cells in (i, j, k) order, in place: an EMPTY cell with at least 5 (3D) or 3 (2D)
 *      FLUID neighbours among its 6 (4) becomes FLUID. In place means that a cell filled earlier in the pass counts
 *      for the cells after it, so the (i-1), (j-1), (k-1) neighbours are read after their own visit.
 * xyz holds count particles as (x, y, z) triples (z unread in 2D); (ox, oy, oz) are FacePos(X|Y|Z, 0), the low face
 * of the first ring cell. Returns the number of particles skipped by ParticleIndex. */
long long or_update_fluid_cells(int dim, int Nx, int Ny, int Nz, double ox, double oy, double oz, double dh,
                                const double *xyz, long long count, uint8_t *types)
{
    const int nz = dim == 3 ? Nz : 1;
    const size_t cells = (size_t)Nx * Ny * nz;
    for (size_t c = 0; c < cells; c++)
    {
        const int t = types[c];
        if (t != SOLID && t != INFLOW && t != OUTFLOW && t != PRESSURE) types[c] = EMPTY;
    }
    long long skipped = 0;
    for (long long p = 0; p < count; p++)
    {
        const int i = ParticleIndex(xyz[3 * p + 1], oy, dh, Ny);
        const int j = ParticleIndex(xyz[3 * p + 0], ox, dh, Nx);
        const int k = dim == 3 ? ParticleIndex(xyz[3 * p + 2], oz, dh, Nz) : 0;
        if (i < 0 || j < 0 || k < 0) { skipped++; continue; }
        const size_t c = ((size_t)i * Nx + j) * nz + k;
        if (types[c] == EMPTY) types[c] = FLUID;
    }
    for (int i = 1; i < Ny - 1; i++)
        for (int j = 1; j < Nx - 1; j++)
        {
            if (dim == 2)
            {
                const size_t c = (size_t)i * Nx + j;
                const int f = (types[c + 1] == FLUID) + (types[c - 1] == FLUID) + (types[c + Nx] == FLUID) +
                              (types[c - Nx] == FLUID);
                if (types[c] == EMPTY && f >= 3) types[c] = FLUID;
                continue;
            }
            for (int k = 1; k < Nz - 1; k++)
            {
                const size_t c = ((size_t)i * Nx + j) * Nz + k, sj = Nz, si = (size_t)Nx * Nz;
                const int f = (types[c + sj] == FLUID) + (types[c - sj] == FLUID) + (types[c + si] == FLUID) +
                              (types[c - si] == FLUID) + (types[c + 1] == FLUID) + (types[c - 1] == FLUID);
                if (types[c] == EMPTY && f >= 5) types[c] = FLUID;
            }
        }
    return skipped;
}

/* MAC::EnforceVelocityBC (src/MAC.cpp:833-858) from the lists MAC::BuildBoundaryLists made, in their order:
 * every solidFaceList[c] entry of field c set to 0; then, when the scene has a boundary velocity function
 * (presc_value not NULL), each prescribedList entry set to its value; then each copyList entry f[dst] = f[src]; then
 * ApplyOutflowFlux (:811-831): with qIn = -sum(sign * f[index] * area) over the inlet faces and qOut =
 * sum(sign * f[index] * area), aOut = sum(area) over the outflow faces, each accumulated in list order,
 * delta = (qIn - qOut) / aOut and each outflow face f[index] += sign * delta, f[outer] = f[index].
 * Fields: comp 0 u, 1 v, 2 w. */
void or_bc_velocity(double *u, double *v, double *w, const int32_t *solid0, const int32_t *solid1,
                    const int32_t *solid2, const int32_t *nsolid, const int32_t *presc_comp,
                    const int32_t *presc_index, const double *presc_value, int npresc, const int32_t *copy_comp,
                    const int32_t *copy_dst, const int32_t *copy_src, int ncopy, const int32_t *in_comp,
                    const int32_t *in_index, const double *in_area, const double *in_sign, int nin,
                    const int32_t *out_comp, const int32_t *out_index, const int32_t *out_outer,
                    const double *out_area, const double *out_sign, int nout)
{
    double *f[3] = {u, v, w};
    const int32_t *solid[3] = {solid0, solid1, solid2};
    for (int c = 0; c < 3; c++)
        for (int q = 0; q < nsolid[c]; q++) f[c][solid[c][q]] = 0.0;
    if (presc_value)
        for (int q = 0; q < npresc; q++) f[presc_comp[q]][presc_index[q]] = presc_value[q];
    for (int q = 0; q < ncopy; q++) f[copy_comp[q]][copy_dst[q]] = f[copy_comp[q]][copy_src[q]];
    if (nout == 0) return;
    double qIn = 0.0, qOut = 0.0, aOut = 0.0;
    for (int q = 0; q < nin; q++) qIn -= in_sign[q] * f[in_comp[q]][in_index[q]] * in_area[q];
    for (int q = 0; q < nout; q++)
    {
        qOut += out_sign[q] * f[out_comp[q]][out_index[q]] * out_area[q];
        aOut += out_area[q];
    }
    if (aOut <= 0.0) return;
    const double delta = (qIn - qOut) / aOut;
    for (int q = 0; q < nout; q++)
    {
        double *g = f[out_comp[q]];
        g[out_index[q]] += out_sign[q] * delta;
        g[out_outer[q]] = g[out_index[q]];
    }
}

/* MAC::EnforcePressureBC (src/MAC.cpp:860-865) from ringList, in order: kind 0 sets p[dst] = 0, kind 1 the
 * prescribed value (value[q], PrescribedPressure at the entry's cell), kind 2 copies p[src]. */
void or_bc_pressure(double *p, const int32_t *dst, const int32_t *kind, const int32_t *src, const double *value,
                    int n)
{
    for (int q = 0; q < n; q++) p[dst[q]] = kind[q] == 0 ? 0.0 : (kind[q] == 1 ? value[q] : p[src[q]]);
}
