// Kernels whose results must match the NEREUS reference bit for bit: scene labelling, IDP numbering, the assembled
// matrix, the right-hand side, the FP64 residual, the scatter and pressure ring, and the projection.
//
// This file is compiled with -fmad=false: every expression rounds after each operation in the order the reference's
// C++ writes it, as the host compiler (which emits no fused multiply-add for the default x86-64 target) does.
#include "nb_kernels.h"

#include <cub/device/device_scan.cuh>

namespace nb
{

// ---------------------------------------------------------------------------------------------------------------
// coefficients, exactly as the reference forms them
// ---------------------------------------------------------------------------------------------------------------

// FaceCoefs3D (PressureSolver3D.cpp:47-63); the 2D c[] table (PressureSolver2D.cpp:123-126).
__device__ __forceinline__ void CoefsExact(const LevelView &v, int i, int j, int k, double c[6])
{
    if (v.dim == 2)
    {
        c[0] = Wd(v, 0, j) / Gp(v, 1, i);
        c[1] = Wd(v, 0, j) / Gp(v, 1, i - 1);
        c[2] = Wd(v, 1, i) / Gp(v, 0, j);
        c[3] = Wd(v, 1, i) / Gp(v, 0, j - 1);
        c[4] = c[5] = 0.0;
        return;
    }
    if (!v.stretched)
    {
        for (int q = 0; q < 6; q++) c[q] = 1.0;
        return;
    }
    const double ax = Wd(v, 1, i) * Wd(v, 2, k);
    const double ay = Wd(v, 0, j) * Wd(v, 2, k);
    const double az = Wd(v, 0, j) * Wd(v, 1, i);
    c[0] = ay / Gp(v, 1, i);
    c[1] = ay / Gp(v, 1, i - 1);
    c[2] = ax / Gp(v, 0, j);
    c[3] = ax / Gp(v, 0, j - 1);
    c[4] = az / Gp(v, 2, k);
    c[5] = az / Gp(v, 2, k - 1);
}

// DirichletRingFactor (PressureSettings.h:307-310).
__device__ __forceinline__ double DRF(const LevelView &v, int a, int n, int s)
{
    return Gp(v, a, s < 0 ? n - 1 : n) / (0.5 * Wd(v, a, n));
}

// RingFactor3D (PressureSolver3D.cpp:80-87) / RingFactor2D (PressureSolver2D.cpp:55-60).
__device__ __forceinline__ double RingFactorExact(const LevelView &v, int i, int j, int k, int q, int t)
{
    if (!IsDirichlet(t)) return 1.0;
    const int ni = i + (q == 0) - (q == 1), nj = j + (q == 2) - (q == 3), nk = k + (q == 4) - (q == 5);
    if (!OnRing(v, ni, nj, nk)) return 1.0;
    const int s = (q % 2 == 0) ? 1 : -1;
    return q < 2 ? DRF(v, 1, i, s) : (q < 4 ? DRF(v, 0, j, s) : DRF(v, 2, k, s));
}

// The diagonal of AssembleSystem before scaling (PressureSolver3D.cpp:151-166): fluid faces first, then the
// Dirichlet faces with their ring factor, in q order. Also reports the neighbour types.
__device__ __forceinline__ double DiagExact(const LevelView &v, int i, int j, int k, long long c, const double cq[6],
                                            int t[6])
{
    const int nq = v.dim == 3 ? 6 : 4;
    double diag = 0.0;
    for (int q = 0; q < nq; q++)
    {
        t[q] = v.types[c + NbrOffset(v, q)];
        if (t[q] == FLUID) diag -= cq[q];
    }
    for (int q = 0; q < nq; q++)
        if (IsDirichlet(t[q])) diag -= cq[q] * RingFactorExact(v, i, j, k, q, t[q]);
    return diag;
}

// ---------------------------------------------------------------------------------------------------------------
// scene labelling: Scene::CellTypeAt (Scene.h:639-673) with Primitive::Distance/Contains (Scene.h:265-366),
// WinningFace (:566-575) and CellTypeOf (:677-686)
// ---------------------------------------------------------------------------------------------------------------
__device__ double PrimDistance(const nb_region &p, int dim, double x, double y, double z)
{
    const int axes = dim == 2 ? 2 : 3;
    double d = 0.0;
    if (p.kind == NB_PRIM_BOX)
    {
        const double c[3] = {x, y, z};
        double outside = 0.0, inside = -1e30;
        for (int a = 0; a < axes; a++)
        {
            const double dlo = p.p0[a] - c[a];
            const double dhi = c[a] - p.p1[a];
            const double dm = dlo > dhi ? dlo : dhi;
            if (dm > 0.0) outside += dm * dm;
            inside = inside > dm ? inside : dm;
        }
        d = outside > 0.0 ? sqrt(outside) : inside;
    }
    else if (p.kind == NB_PRIM_SPHERE)
    {
        const double dx = x - p.p0[0], dy = y - p.p0[1];
        const double dz = axes == 3 ? (z - p.p0[2]) : 0.0;
        d = sqrt(dx * dx + dy * dy + dz * dz) - p.radius;
    }
    else if (p.kind == NB_PRIM_CYLINDER)
    {
        double a1, a2;
        if (p.axis == 0) { a1 = y - p.p0[1]; a2 = z - p.p0[2]; }
        else if (p.axis == 1) { a1 = x - p.p0[0]; a2 = z - p.p0[2]; }
        else { a1 = x - p.p0[0]; a2 = y - p.p0[1]; }
        d = sqrt(a1 * a1 + a2 * a2) - p.radius;
    }
    else
    {
        const double nx = p.p1[0], ny = p.p1[1];
        const double nz = axes == 3 ? p.p1[2] : 0.0;
        const double len = sqrt(nx * nx + ny * ny + nz * nz);
        const double inv = len > 0.0 ? 1.0 / len : 0.0;
        const double dzc = axes == 3 ? (z - p.p0[2]) : 0.0;
        d = ((x - p.p0[0]) * nx + (y - p.p0[1]) * ny + dzc * nz) * inv;
    }
    return p.invert ? -d : d;
}

__global__ void k_label_cells(int dim, int Nx, int Ny, int Nz, const double *cx, const double *cy, const double *cz,
                              nb_scene s, uint8_t *types)
{
    const long long cells = (long long)Nx * Ny * Nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells;
         c += (long long)gridDim.x * blockDim.x)
    {
        const int k = (int)(c % Nz);
        const long long r = c / Nz;
        const int j = (int)(r % Nx), i = (int)(r / Nx);
        const double x = cx[j], y = cy[i], z = dim == 3 ? cz[k] : cz[0];
        int type = FLUID;
        for (int q = 0; q < s.nregions; q++)
        {
            const nb_region &p = s.regions[q];
            if (!(PrimDistance(p, dim, x, y, z) < 0.0)) continue;
            type = p.region == NB_REGION_SOLID ? SOLID : (p.region == NB_REGION_FLUID ? FLUID : EMPTY);
        }
        const bool on[6] = {j == 0, j == Nx - 1, i == 0, i == Ny - 1, k == 0, k == Nz - 1};
        int best = -1, bestOrder = -2;
        for (int f = 0; f < 6; f++)
        {
            if (!on[f] || (dim == 2 && f >= 4)) continue;
            if (s.face_order[f] > bestOrder) { bestOrder = s.face_order[f]; best = f; }
        }
        if (best >= 0)
        {
            const int kind = s.face_kind[best];
            type = kind == NB_BC_INLET ? INFLOW
                 : kind == NB_BC_OUTFLOW ? OUTFLOW
                 : kind == NB_BC_PRESSURE_OUTLET ? (s.face_has_p[best] ? PRESSURE : EMPTY) : SOLID;
        }
        types[c] = (uint8_t)type;
    }
}

void LaunchLabelCells(int dim, int Nx, int Ny, int Nz, const double *cx, const double *cy, const double *cz,
                      const nb_scene &s, uint8_t *types, cudaStream_t st)
{
    const long long cells = (long long)Nx * Ny * Nz;
    int blocks = (int)((cells + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    NB_COUNT_LAUNCH();
    k_label_cells<<<blocks, 256, 0, st>>>(dim, Nx, Ny, Nz, cx, cy, cz, s, types);
}

// ---------------------------------------------------------------------------------------------------------------
// IDP numbering (PressureSolver3D.cpp:133-139): interior FLUID cells in (i, j, k) order = the order of lines, then
// the fast axis. Count per line, exclusive scan, then a warp-ballot prefix inside each line.
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_line_counts(LevelView v, int *counts)
{
    const int lane = threadIdx.x & 31, warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int line = warp; line < v.nLines; line += nw)
    {
        int cnt = 0;
        for (int f0 = 0; f0 < v.lineLen; f0 += 32)
        {
            const int f = f0 + lane;
            int i, j, k;
            long long c;
            LineCell(v, line, f < v.lineLen ? f : 0, i, j, k, c);
            const bool fl = f < v.lineLen && v.types[c] == FLUID;
            cnt += __popc(__ballot_sync(0xffffffffu, fl));
        }
        if (lane == 0) counts[line] = cnt;
    }
}

__global__ void k_line_number(LevelView v, const int *offsets, int32_t *idp)
{
    const int lane = threadIdx.x & 31, warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int line = warp; line < v.nLines; line += nw)
    {
        int base = offsets[line];
        for (int f0 = 0; f0 < v.lineLen; f0 += 32)
        {
            const int f = f0 + lane;
            int i, j, k;
            long long c;
            LineCell(v, line, f < v.lineLen ? f : 0, i, j, k, c);
            const bool fl = f < v.lineLen && v.types[c] == FLUID;
            const unsigned m = __ballot_sync(0xffffffffu, fl);
            if (fl) idp[c] = base + __popc(m & ((1u << lane) - 1u));
            base += __popc(m);
        }
    }
}

int NumberUnknowns(const LevelView &v, int32_t *idp, int *lineCounts, int *lineOffsets, void *scanTmp,
                   size_t scanTmpBytes, int *hostTotal, cudaStream_t st)
{
    cudaMemsetAsync(idp, 0xFF, sizeof(int32_t) * (size_t)v.cells, st);
    if (v.nLines <= 0 || v.lineLen <= 0) { *hostTotal = 0; return 0; }
    const int blocks = LineGrid(v.nLines, 148 * 8);
    NB_COUNT_LAUNCH();
    k_line_counts<<<blocks, kBlock, 0, st>>>(v, lineCounts);
    size_t bytes = scanTmpBytes;
    cub::DeviceScan::ExclusiveSum(scanTmp, bytes, lineCounts, lineOffsets, v.nLines + 1, st);
    NB_COUNT_LAUNCH();
    k_line_number<<<blocks, kBlock, 0, st>>>(v, lineOffsets, idp);
    int total = 0;
    cudaMemcpyAsync(&total, lineOffsets + v.nLines, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    *hostTotal = total;
    return 0;
}

size_t ScanTempBytes(int n)
{
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (int *)nullptr, (int *)nullptr, n, (cudaStream_t)0);
    return bytes;
}

// ---------------------------------------------------------------------------------------------------------------
// the assembled matrix, exported as CSR (AssembleSystem + setFromTriplets): row lengths, scan, fill
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_row_lengths(LevelView v, const int32_t *idp, int *rowLen, int *dirichletFlag)
{
    const int lane = threadIdx.x & 31, warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    int dir = 0;
    for (int line = warp; line < v.nLines; line += nw)
        for (int f = lane; f < v.lineLen; f += 32)
        {
            int i, j, k;
            long long c;
            LineCell(v, line, f, i, j, k, c);
            const int row = idp[c];
            if (row < 0) continue;
            double cq[6];
            int t[6];
            CoefsExact(v, i, j, k, cq);
            const double diag = DiagExact(v, i, j, k, c, cq, t);
            int len = diag != 0.0 ? 1 : 0;
            const int nq = v.dim == 3 ? 6 : 4;
            for (int q = 0; q < nq; q++)
            {
                if (t[q] == FLUID)
                {
                    if (idp[c + NbrOffset(v, q)] >= 0) len++;
                    else dir = 1;
                }
                if (IsDirichlet(t[q])) dir = 1;
            }
            rowLen[row] = len;
        }
    if (dir) atomicOr(dirichletFlag, 1);
}

__global__ void k_row_fill(LevelView v, const int32_t *idp, const int *rowPtr, int32_t *col, double *val, double scale)
{
    const int lane = threadIdx.x & 31, warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    // ascending column order = ascending linear offset: i-1, j-1, k-1, diagonal, k+1, j+1, i+1
    const int order3[7] = {1, 3, 5, -1, 4, 2, 0};
    const int order2[5] = {1, 3, -1, 2, 0};
    for (int line = warp; line < v.nLines; line += nw)
        for (int f = lane; f < v.lineLen; f += 32)
        {
            int i, j, k;
            long long c;
            LineCell(v, line, f, i, j, k, c);
            const int row = idp[c];
            if (row < 0) continue;
            double cq[6];
            int t[6];
            CoefsExact(v, i, j, k, cq);
            const double diag = DiagExact(v, i, j, k, c, cq, t);
            int e = rowPtr[row];
            const int ne = v.dim == 3 ? 7 : 5;
            for (int s = 0; s < ne; s++)
            {
                const int q = v.dim == 3 ? order3[s] : order2[s];
                if (q < 0)
                {
                    if (diag != 0.0) { col[e] = row; val[e] = scale * diag; e++; }
                    continue;
                }
                if (t[q] != FLUID) continue;
                const int cl = idp[c + NbrOffset(v, q)];
                if (cl < 0) continue;
                col[e] = cl;
                val[e] = scale * cq[q];
                e++;
            }
        }
}

int ExportMatrix(const LevelView &v, const int32_t *idp, int n, double scale, int *rowLen, int *rowPtr,
                 int32_t *col, double *val, int *flag, void *scanTmp, size_t scanTmpBytes, int *hostNnz,
                 int *hostSingular, cudaStream_t st)
{
    cudaMemsetAsync(flag, 0, sizeof(int), st);
    cudaMemsetAsync(rowLen, 0, sizeof(int) * (size_t)(n + 1), st);
    const int blocks = LineGrid(v.nLines, 148 * 8);
    if (v.nLines > 0)
    {
        NB_COUNT_LAUNCH();
        k_row_lengths<<<blocks, kBlock, 0, st>>>(v, idp, rowLen, flag);
    }
    size_t bytes = scanTmpBytes;
    cub::DeviceScan::ExclusiveSum(scanTmp, bytes, rowLen, rowPtr, n + 1, st);
    if (v.nLines > 0 && n > 0)
    {
        NB_COUNT_LAUNCH();
        k_row_fill<<<blocks, kBlock, 0, st>>>(v, idp, rowPtr, col, val, scale);
    }
    int nnz = 0, dir = 0;
    cudaMemcpyAsync(&nnz, rowPtr + n, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&dir, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    *hostNnz = nnz;
    *hostSingular = dir ? 0 : 1;
    return 0;
}

// ---------------------------------------------------------------------------------------------------------------
// divergence and right-hand side: MAC::GetDivergencyAt (src/MAC.cpp:349-367, 443-456), DirichletSum
// (PressureSolver3D.cpp:248-260) and SolveScheme's loop (:288-298)
// ---------------------------------------------------------------------------------------------------------------
struct Faces
{
    const double *u, *v, *w;
    long long uI, uJ, vI, vJ, wI, wJ; // strides of i and j in u, v, w (k stride 1)
};

__device__ __forceinline__ double DivergenceAt(const LevelView &g, const Faces &F, int i, int j, int k, double dh)
{
    const long long cu = i * F.uI + j * F.uJ + k, cv = i * F.vI + j * F.vJ + k;
    if (g.dim == 2)
    {
        if (g.stretched)
        {
            const double dx = Wd(g, 0, j), dy = Wd(g, 1, i);
            const double fluxU = (F.u[cu + F.uJ] - F.u[cu]) * dy;
            const double fluxV = (F.v[cv + F.vI] - F.v[cv]) * dx;
            return (fluxU + fluxV) / (dx * dy);
        }
        const double divU = (F.u[cu + F.uJ] - F.u[cu]) / dh;
        const double divV = (F.v[cv + F.vI] - F.v[cv]) / dh;
        return divU + divV;
    }
    const long long cw = i * F.wI + j * F.wJ + k;
    if (g.stretched)
    {
        const double dx = Wd(g, 0, j), dy = Wd(g, 1, i), dz = Wd(g, 2, k);
        const double fluxU = (F.u[cu + F.uJ] - F.u[cu]) * dy * dz;
        const double fluxV = (F.v[cv + F.vI] - F.v[cv]) * dx * dz;
        const double fluxW = (F.w[cw + 1] - F.w[cw]) * dx * dy;
        return (fluxU + fluxV + fluxW) / (dx * dy * dz);
    }
    const double divU = (F.u[cu + F.uJ] - F.u[cu]) / dh;
    const double divV = (F.v[cv + F.vI] - F.v[cv]) / dh;
    const double divW = (F.w[cw + 1] - F.w[cw]) / dh;
    return divU + divV + divW;
}

__global__ void k_rhs(LevelView v, Faces F, const double *p, double rhoDt, double scale, double dh, double *b)
{
    const int fo = blockIdx.x * kTileF + threadIdx.x, mo = blockIdx.y * kTileM + threadIdx.y;
    const int sBeg = blockIdx.z * v.slowChunk, sEnd = min(sBeg + v.slowChunk, v.slowLen);
    for (int s = sBeg; s < sEnd; s++)
        {
            int i, j, k;
            long long c;
            if (!TileCell(v, fo, mo, s, i, j, k, c)) continue;
            const unsigned code = v.code[c];
            if (!(code & CODE_UNKNOWN)) continue; // an interior FLUID cell
            double ds = 0.0;
            if (code & CODE_DIRICHLET) // a PRESSURE neighbour is a Dirichlet one: the others skip the scan
            {
                double cq[6];
                CoefsExact(v, i, j, k, cq);
                const int nq = v.dim == 3 ? 6 : 4;
                for (int q = 0; q < nq; q++)
                {
                    const long long n = c + NbrOffset(v, q);
                    const int t = v.types[n];
                    if (t == PRESSURE) ds += cq[q] * RingFactorExact(v, i, j, k, q, t) * p[n];
                }
            }
            double vol = 1.0;
            if (v.stretched) vol = v.dim == 3 ? Wd(v, 0, j) * Wd(v, 1, i) * Wd(v, 2, k) : Wd(v, 0, j) * Wd(v, 1, i);
            b[c] = rhoDt * DivergenceAt(v, F, i, j, k, dh) * vol - scale * ds;
        }
}

// The same right-hand side on a uniform 3D grid with Nz even, two cells along k per thread (nb_device.cuh, PairPos):
// the u faces of a pair are one aligned 16-byte load per row (u rows have Nz entries), the v faces one per plane (the
// v plane of i+1 is kept for the next step of the march), the w faces three scalars (w rows have Nz+1 entries). Each
// cell's expression is k_rhs's, operation for operation.
__global__ void __launch_bounds__(kPairThreads, 4) k_pair_rhs(LevelView v, Faces F, const double *p, double rhoDt,
                                                           double scale, double dh, double *b)
{
    const PairPos P = PairStart(v);
    const long long uPlane = F.uI, wPlane = F.wI;
    const int Nz = v.Nz;
    // plane i's v faces (i, j, k) are the pair at the cell index; (i+1, j, k) one plane on
    double2 vC = *reinterpret_cast<const double2 *>(F.v + P.base);
    int off = 0;
    for (int i = P.i0; i < P.i1; i++, off += P.sI)
    {
        const long long c = P.base + off;
        const long long cu = (long long)i * uPlane + (long long)P.j * Nz + P.k0;
        const long long cw = (long long)i * wPlane + (long long)P.j * (Nz + 1) + P.k0;
        const double2 u0 = *reinterpret_cast<const double2 *>(F.u + cu);
        const double2 u1 = *reinterpret_cast<const double2 *>(F.u + cu + Nz);
        const double2 vP = *reinterpret_cast<const double2 *>(F.v + c + P.sI);
        const double w0 = F.w[cw], w1 = F.w[cw + 1], w2 = F.w[cw + 2];
        const unsigned code2 = *reinterpret_cast<const unsigned short *>(v.code + c);
        if (P.valid && (code2 & ((unsigned)CODE_UNKNOWN | ((unsigned)CODE_UNKNOWN << 8))))
        {
            double out[2];
#pragma unroll
            for (int h = 0; h < 2; h++)
            {
                const unsigned code = (code2 >> (8 * h)) & 0xFFu;
                out[h] = 0.0;
                if (!(code & CODE_UNKNOWN)) continue;
                const int k = P.k0 + h;
                double ds = 0.0;
                if (code & CODE_DIRICHLET)
                {
                    double cq[6];
                    CoefsExact(v, i, P.j, k, cq);
                    for (int q = 0; q < 6; q++)
                    {
                        const long long n = c + h + NbrOffset(v, q);
                        const int t = v.types[n];
                        if (t == PRESSURE) ds += cq[q] * RingFactorExact(v, i, P.j, k, q, t) * p[n];
                    }
                }
                const double divU = ((h ? u1.y : u1.x) - (h ? u0.y : u0.x)) / dh;
                const double divV = ((h ? vP.y : vP.x) - (h ? vC.y : vC.x)) / dh;
                const double divW = ((h ? w2 : w1) - (h ? w1 : w0)) / dh;
                const double vol = 1.0;
                out[h] = rhoDt * (divU + divV + divW) * vol - scale * ds;
            }
            *reinterpret_cast<double2 *>(b + c) = make_double2(out[0], out[1]);
        }
        vC = vP;
    }
}

Faces MakeFaces(const LevelView &v, const double *u, const double *vv, const double *w)
{
    Faces F;
    F.u = u; F.v = vv; F.w = w;
    const long long Nx = v.Nx, Ny = v.Ny, Nz = v.Nz;
    (void)Ny;
    F.uJ = Nz; F.uI = (Nx + 1) * Nz;
    F.vJ = Nz; F.vI = Nx * Nz;
    F.wJ = Nz + 1; F.wI = Nx * (Nz + 1);
    return F;
}

void LaunchRhs(const LevelView &v, const double *u, const double *vv, const double *w, const double *p, double rhoDt,
               double scale, double dh, double *b, cudaStream_t st)
{
    if (v.nLines <= 0) return;
    NB_COUNT_LAUNCH();
    if (v.dim == 3 && !v.stretched && v.Nz % 2 == 0 && v.code)
        k_pair_rhs<<<PairGrid(v), kPairThreads, 0, st>>>(v, MakeFaces(v, u, vv, w), p, rhoDt, scale, dh, b);
    else
        k_rhs<<<TileGrid(v), dim3(kTileF, kTileM), 0, st>>>(v, MakeFaces(v, u, vv, w), p, rhoDt, scale, dh, b);
}

// max |div u| over FLUID cells (the post-projection check)
__global__ void k_max_div(LevelView v, Faces F, double dh, Reducer R, int slot)
{
    const int fo = blockIdx.x * kTileF + threadIdx.x, mo = blockIdx.y * kTileM + threadIdx.y;
    const int sBeg = blockIdx.z * v.slowChunk, sEnd = min(sBeg + v.slowChunk, v.slowLen);
    double m[1] = {0.0};
    for (int s = sBeg; s < sEnd; s++)
        {
            int i, j, k;
            long long c;
            if (!TileCell(v, fo, mo, s, i, j, k, c)) continue;
            if (v.types[c] != FLUID) continue;
            m[0] = fmax(m[0], fabs(DivergenceAt(v, F, i, j, k, dh)));
        }
    GridReduce<1>(R, m, slot, 1);
}

// The same check on a uniform 3D grid with Nz even, two cells per thread (the face loads of k_pair_rhs).
__global__ void __launch_bounds__(kPairThreads) k_pair_max_div(LevelView v, Faces F, double dh, Reducer R, int slot)
{
    const PairPos P = PairStart(v);
    const int Nz = v.Nz;
    double m[1] = {0.0};
    double2 vC = *reinterpret_cast<const double2 *>(F.v + P.base);
    int off = 0;
    for (int i = P.i0; i < P.i1; i++, off += P.sI)
    {
        const long long c = P.base + off;
        const long long cu = (long long)i * F.uI + (long long)P.j * Nz + P.k0;
        const long long cw = (long long)i * F.wI + (long long)P.j * (Nz + 1) + P.k0;
        const double2 u0 = *reinterpret_cast<const double2 *>(F.u + cu);
        const double2 u1 = *reinterpret_cast<const double2 *>(F.u + cu + Nz);
        const double2 vP = *reinterpret_cast<const double2 *>(F.v + c + P.sI);
        const double w0 = F.w[cw], w1 = F.w[cw + 1], w2 = F.w[cw + 2];
        const unsigned code2 = *reinterpret_cast<const unsigned short *>(v.code + c);
        if (P.valid)
        {
            if (code2 & CODE_UNKNOWN)
            {
                const double d = (u1.x - u0.x) / dh + (vP.x - vC.x) / dh + (w1 - w0) / dh;
                m[0] = fmax(m[0], fabs(d));
            }
            if ((code2 >> 8) & CODE_UNKNOWN)
            {
                const double d = (u1.y - u0.y) / dh + (vP.y - vC.y) / dh + (w2 - w1) / dh;
                m[0] = fmax(m[0], fabs(d));
            }
        }
        vC = vP;
    }
    GridReduce<1>(R, m, slot, 1);
}

void LaunchMaxDiv(const LevelView &v, const double *u, const double *vv, const double *w, double dh,
                  const Reducer &R, int slot, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    if (v.dim == 3 && !v.stretched && v.Nz % 2 == 0 && v.code && v.Ny >= 3)
        k_pair_max_div<<<PairGrid(v, 16), kPairThreads, 0, st>>>(v, MakeFaces(v, u, vv, w), dh, R, slot);
    else
        k_max_div<<<TileGrid(v), dim3(kTileF, kTileM), 0, st>>>(v, MakeFaces(v, u, vv, w), dh, R, slot);
}

// ---------------------------------------------------------------------------------------------------------------
// The incremental scheme's cell-by-cell steps and the warm start's guess, each the reference's expression:
//   CELL_DELTA      out = a - b on PRESSURE cells, 0 elsewhere: DirichletSum's known value p_b(t^{n+1}) - p_b(t^n)
//                   (PressureSolver3D.cpp:248-260, `old` non-null)
//   CELL_RING_DELTA a -= b on PRESSURE cells: the increment's ring after EnforcePressureBC (:321-328)
//   CELL_NEG        out = -a on the unknowns, 0 elsewhere: b + A p^n = b - A(-p^n) (IncrementReferenceNorm :262-276)
//   CELL_TAKE       out = a on the unknowns, 0 elsewhere: BuildWarmStartGuess's x0 (:222-244)
//   CELL_SUM        out = a + b on the unknowns, 0 elsewhere: p^n + phi (AccumulatePressureIncrement :374-393)
//   CELL_RESTORE    a = b on PRESSURE cells: the prescribed ring p_b(t^{n+1}) put back (EnforcePressureBC)
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_cellwise(LevelView v, int op, double *a, const double *b, double *out)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < v.cells;
         c += (long long)gridDim.x * blockDim.x)
    {
        const int t = v.types[c];
        bool unknown = false;
        if (op == CELL_NEG || op == CELL_TAKE || op == CELL_SUM)
        {
            const int k = v.dim == 3 ? (int)(c % v.Nz) : 1;
            const long long rr = v.dim == 3 ? c / v.Nz : c;
            const int j = (int)(rr % v.Nx), i = (int)(rr / v.Nx);
            unknown = t == FLUID && i > 0 && i < v.Ny - 1 && j > 0 && j < v.Nx - 1 &&
                      (v.dim == 2 || (k > 0 && k < v.Nz - 1));
        }
        switch (op)
        {
        case CELL_DELTA: out[c] = t == PRESSURE ? a[c] - b[c] : 0.0; break;
        case CELL_RING_DELTA: if (t == PRESSURE) a[c] = a[c] - b[c]; break;
        case CELL_NEG: out[c] = unknown ? -a[c] : 0.0; break;
        case CELL_TAKE: out[c] = unknown ? a[c] : 0.0; break;
        case CELL_SUM: out[c] = unknown ? a[c] + b[c] : 0.0; break;
        case CELL_RESTORE: if (t == PRESSURE) a[c] = b[c]; break;
        default: break;
        }
    }
}

void LaunchCellwise(const LevelView &v, int op, double *a, const double *b, double *out, cudaStream_t st)
{
    int blocks = (int)((v.cells + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    NB_COUNT_LAUNCH();
    k_cellwise<<<blocks, 256, 0, st>>>(v, op, a, b, out);
}

// ---------------------------------------------------------------------------------------------------------------
// FP64 residual of the reference's matrix: r = b - A x, A = scale * (off-diagonals c_q, diagonal DiagExact).
// Writes the unit-form residual -r/scale in T for the solver, sums ||r||^2 (and r for a singular system).
// The refinement form also adds a correction e first: x_out = x_in + e, r = b - A x_out, read from the
// neighbours' x_in + e, so x_in and x_out are different arrays.
// ---------------------------------------------------------------------------------------------------------------
// swap (refinement form, may be null): when *swap is odd, x_in and x_out trade places (a refinement loop on the device
// alternates its two iterates without the host)
template <typename T, bool kAdd>
__global__ void k_residual64(LevelView v, const double *b, const double *xin0, const T *e, double *xout0, T *rOut,
                             double scale, double sfac, Reducer R, int slot, const int *swap)
{
    const bool sw = kAdd && swap && (*swap & 1);
    const double *xin = sw ? xout0 : xin0;
    double *xout = sw ? const_cast<double *>(xin0) : xout0;
    const int fo = blockIdx.x * kTileF + threadIdx.x, mo = blockIdx.y * kTileM + threadIdx.y;
    const int sBeg = blockIdx.z * v.slowChunk, sEnd = min(sBeg + v.slowChunk, v.slowLen);
    double acc[2] = {0.0, 0.0};
    for (int s = sBeg; s < sEnd; s++)
        {
            int i, j, k;
            long long c;
            if (!TileCell(v, fo, mo, s, i, j, k, c)) continue;
            if (v.types[c] != FLUID) continue;
            double cq[6];
            int t[6];
            CoefsExact(v, i, j, k, cq);
            const double diag = DiagExact(v, i, j, k, c, cq, t);
            // e and rOut are level vectors: the grid layout, or the colour-split one of a split level 0
            const double xc = kAdd ? xin[c] + (double)e[VecIdx(v, i, j, k)] : xin[c];
            double off = 0.0;
            const int nq = v.dim == 3 ? 6 : 4;
            for (int q = 0; q < nq; q++)
                if (t[q] == FLUID)
                {
                    const long long n = c + NbrOffset(v, q);
                    const int ni = i + (q == 0) - (q == 1), nj = j + (q == 2) - (q == 3), nk = k + (q == 4) - (q == 5);
                    const double xn = kAdd ? xin[n] + (double)e[VecIdx(v, ni, nj, nk)] : xin[n];
                    off += cq[q] * xn;
                }
            const double ax = scale * (off + diag * xc);
            const double r = b[c] - ax;
            if (kAdd) xout[c] = xc;
            rOut[VecIdx(v, i, j, k)] = (T)(r * sfac);
            acc[0] += r * r;
            acc[1] += r;
        }
    GridReduce<2>(R, acc, slot);
}

template <typename T>
void LaunchResidual64(const LevelView &v, const double *b, const double *x, T *rOut, double scale, double sfac,
                      const Reducer &R, int slot, cudaStream_t st)
{
    const int blocks = LineGrid(v.nLines > 0 ? v.nLines : 1, R.maxBlocks);
    NB_COUNT_LAUNCH();
    k_residual64<T, false><<<TileGrid(v), dim3(kTileF, kTileM), 0, st>>>(v, b, x, (const T *)nullptr, nullptr, rOut,
                                                                          scale, sfac, R, slot, nullptr);
}

template <typename T>
void LaunchRefine64(const LevelView &v, const double *b, const double *xin, const T *e, double *xout, T *rOut,
                    double scale, double sfac, const Reducer &R, int slot, cudaStream_t st, const int *swap)
{
    NB_COUNT_LAUNCH();
    k_residual64<T, true><<<TileGrid(v), dim3(kTileF, kTileM), 0, st>>>(v, b, xin, e, xout, rOut, scale, sfac, R, slot,
                                                                         swap);
}

template void LaunchResidual64<float>(const LevelView &, const double *, const double *, float *, double, double,
                                      const Reducer &, int, cudaStream_t);
template void LaunchResidual64<double>(const LevelView &, const double *, const double *, double *, double, double,
                                       const Reducer &, int, cudaStream_t);
template void LaunchRefine64<float>(const LevelView &, const double *, const double *, const float *, double *,
                                    float *, double, double, const Reducer &, int, cudaStream_t, const int *);
template void LaunchRefine64<double>(const LevelView &, const double *, const double *, const double *, double *,
                                     double *, double, double, const Reducer &, int, cudaStream_t, const int *);

// ---------------------------------------------------------------------------------------------------------------
// level, scatter, ring (PressureSolver3D.cpp:181-187, 321-328; MAC::EnforcePressureBC src/MAC.cpp:866-871 replaying
// BuildRingList :1064-1096 -- y faces, then x, then z; EMPTY 0, PRESSURE kept, any other ring cell copies inward)
// ---------------------------------------------------------------------------------------------------------------

// sum of x over the unknowns, compensated (Neumaier) per thread, then the deterministic reduction of (sum, carry)
__global__ void k_sum_unknowns(LevelView v, const double *x, Reducer R, int slot)
{
    const int fo = blockIdx.x * kTileF + threadIdx.x, mo = blockIdx.y * kTileM + threadIdx.y;
    const int sBeg = blockIdx.z * v.slowChunk, sEnd = min(sBeg + v.slowChunk, v.slowLen);
    double sum = 0.0, comp = 0.0;
    for (int s = sBeg; s < sEnd; s++)
    {
        int i, j, k;
        long long c;
        if (!TileCell(v, fo, mo, s, i, j, k, c)) continue;
        if (v.types[c] != FLUID) continue;
        const double a = x[c];
        const double t = sum + a;
        comp += fabs(sum) >= fabs(a) ? (sum - t) + a : (a - t) + sum;
        sum = t;
    }
    double acc[2] = {sum, comp};
    GridReduce<2>(R, acc, slot);
}

// x -= (out[slot] + out[slot+1]) / n at the unknowns, then optionally scatter into p.
__global__ void k_sub_mean_scatter(LevelView v, double *x, const double *sums, int n, int sub, double *p)
{
    const int fo = blockIdx.x * kTileF + threadIdx.x, mo = blockIdx.y * kTileM + threadIdx.y;
    const int sBeg = blockIdx.z * v.slowChunk, sEnd = min(sBeg + v.slowChunk, v.slowLen);
    const double mean = sub ? (sums[0] + sums[1]) / (double)n : 0.0;
    for (int s = sBeg; s < sEnd; s++)
        {
            int i, j, k;
            long long c;
            if (!TileCell(v, fo, mo, s, i, j, k, c)) continue;
            if (v.types[c] != FLUID) continue;
            const double y = x[c] - mean;
            x[c] = y;
            if (p) p[c] = y;
        }
}

void LaunchSumUnknowns(const LevelView &v, const double *x, const Reducer &R, int slot, cudaStream_t st)
{
    const int blocks = LineGrid(v.nLines > 0 ? v.nLines : 1, R.maxBlocks);
    NB_COUNT_LAUNCH();
    k_sum_unknowns<<<TileGrid(v), dim3(kTileF, kTileM), 0, st>>>(v, x, R, slot);
}

// The same over the whole array in order, the unknowns told by their code byte (interior FLUID cells).
__global__ void __launch_bounds__(256) k_lin_sub_mean_scatter(long long cells, const uint8_t *__restrict__ code,
                                                              double *x, const double *sums, int n, int sub,
                                                              double *p)
{
    const double mean = sub ? (sums[0] + sums[1]) / (double)n : 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cells;
         t += (long long)gridDim.x * blockDim.x)
    {
        if (!(code[t] & CODE_UNKNOWN)) continue;
        const double y = x[t] - mean;
        if (sub) x[t] = y;
        if (p) p[t] = y;
    }
}

void LaunchSubMeanScatter(const LevelView &v, double *x, const double *sums, int n, int sub, double *p, cudaStream_t st)
{
    if (v.nLines <= 0) return;
    NB_COUNT_LAUNCH();
    if (v.code)
        k_lin_sub_mean_scatter<<<148 * 8, 256, 0, st>>>(v.cells, v.code, x, sums, n, sub, p);
    else
        k_sub_mean_scatter<<<TileGrid(v), dim3(kTileF, kTileM), 0, st>>>(v, x, sums, n, sub, p);
}

__device__ __forceinline__ void RingEntry(const LevelView &v, double *p, long long d, long long s)
{
    const int t = v.types[d];
    if (t == EMPTY) p[d] = 0.0;
    else if (t != PRESSURE) p[d] = p[s];
}

// pass 0: y faces (i = 0, Ny-1) over (j, k); pass 1: x faces (j = 0, Nx-1) over (i, k); pass 2: z faces over (i, j)
__global__ void k_ring(LevelView v, double *p, int pass)
{
    const int Nx = v.Nx, Ny = v.Ny, Nz = v.Nz;
    const long long A = pass == 0 ? Nx : Ny;
    const long long B = pass == 2 ? Nx : Nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < A * B;
         t += (long long)gridDim.x * blockDim.x)
    {
        const int a = (int)(t / B), b = (int)(t % B);
        long long lo, loSrc, hi, hiSrc;
        if (pass == 0)
        {
            lo = (long long)a * v.sJ + b; loSrc = lo + v.sI;
            hi = (long long)(Ny - 1) * v.sI + lo; hiSrc = hi - v.sI;
        }
        else if (pass == 1)
        {
            lo = (long long)a * v.sI + b; loSrc = lo + v.sJ;
            hi = lo + (long long)(Nx - 1) * v.sJ; hiSrc = hi - v.sJ;
        }
        else
        {
            lo = (long long)a * v.sI + (long long)b * v.sJ; loSrc = lo + 1;
            hi = lo + (Nz - 1); hiSrc = hi - 1;
        }
        RingEntry(v, p, lo, loSrc);
        RingEntry(v, p, hi, hiSrc);
    }
}

void LaunchRing(const LevelView &v, double *p, cudaStream_t st)
{
    const int passes = v.dim == 3 ? 3 : 2;
    for (int pass = 0; pass < passes; pass++)
    {
        const long long A = pass == 0 ? v.Nx : v.Ny;
        const long long B = pass == 2 ? v.Nx : v.Nz;
        int blocks = (int)((A * B + 255) / 256);
        if (blocks > 148 * 4) blocks = 148 * 4;
        if (blocks < 1) blocks = 1;
        NB_COUNT_LAUNCH();
        k_ring<<<blocks, 256, 0, st>>>(v, p, pass);
    }
}

// ---------------------------------------------------------------------------------------------------------------
// the projection: ProjectPressure (PressureSolver3D.cpp:417-438; 2D :382-395), ProjectionGradient
// (PressureSolver3D.cpp:405-414; 2D :370-379), MAC::GetGradP (MAC.h:149-154) and FaceGate (MAC.h:271-274):
// u -= dt/rho * grad p on every face whose two cells are not SOLID. One thread per cell (i, j, k) updates the
// low u, v, w faces of that cell that lie in their component's loop range.
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ double ProjGrad(const LevelView &g, int a, int i, int j, int k, long long c, const double *p)
{
    double grad;
    if (a == 0) grad = (p[c] - p[c - g.sJ]) / Gp(g, 0, j - 1);
    else if (a == 1) grad = (p[c] - p[c - g.sI]) / Gp(g, 1, i - 1);
    else grad = (p[c] - p[c - 1]) / Gp(g, 2, k - 1);
    const int n = a == 0 ? j : (a == 1 ? i : k);
    const int N = a == 0 ? g.Nx : (a == 1 ? g.Ny : g.Nz);
    if (g.dim == 2)
    {
        if (n == 1 && IsDirichlet(a == 0 ? g.types[(long long)i * g.sI] : g.types[(long long)j * g.sJ]))
            return grad * DRF(g, a, 1, -1);
        if (n == N - 1 && IsDirichlet(a == 0 ? g.types[(long long)i * g.sI + (long long)(N - 1) * g.sJ]
                                             : g.types[(long long)(N - 1) * g.sI + (long long)j * g.sJ]))
            return grad * DRF(g, a, N - 2, +1);
        return grad;
    }
    if (n != 1 && n != N - 1) return grad;
    const int r = n == 1 ? 0 : N - 1;
    const long long rc = a == 0 ? (long long)i * g.sI + (long long)r * g.sJ + k
                       : (a == 1 ? (long long)r * g.sI + (long long)j * g.sJ + k
                                 : (long long)i * g.sI + (long long)j * g.sJ + r);
    if (!IsDirichlet(g.types[rc])) return grad;
    return n == 1 ? grad * DRF(g, a, 1, -1) : grad * DRF(g, a, N - 2, +1);
}

__global__ void k_project(LevelView g, double *u, double *v, double *w, const double *p, double f)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x + (g.dim == 3 ? 1 : 0);
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int i = blockIdx.z + 1;
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
    const int kEnd = g.dim == 3 ? Nz : 1; // w faces run to Nz-1; u, v stop at Nz-2
    if (j > Nx - 1 || i > Ny - 1 || k >= kEnd) return;
    const long long c = (long long)i * g.sI + (long long)j * g.sJ + k;
    const int tc = g.types[c];
    const bool kIn = g.dim == 2 || k <= Nz - 2;
    // u face (i, j, k): i in [1, Ny-2], j in [1, Nx-1], k in [1, Nz-2]
    if (i <= Ny - 2 && kIn)
    {
        if (!(tc == SOLID || g.types[c - g.sJ] == SOLID))
        {
            const long long fu = ((long long)i * (Nx + 1) + j) * Nz + k;
            u[fu] = u[fu] - f * ProjGrad(g, 0, i, j, k, c, p);
        }
    }
    // v face: i in [1, Ny-1], j in [1, Nx-2]
    if (j <= Nx - 2 && kIn)
    {
        if (!(tc == SOLID || g.types[c - g.sI] == SOLID))
        {
            const long long fv = ((long long)i * Nx + j) * Nz + k;
            v[fv] = v[fv] - f * ProjGrad(g, 1, i, j, k, c, p);
        }
    }
    // w face: i in [1, Ny-2], j in [1, Nx-2], k in [1, Nz-1]
    if (g.dim == 3 && i <= Ny - 2 && j <= Nx - 2)
    {
        if (!(tc == SOLID || g.types[c - 1] == SOLID))
        {
            const long long fw = ((long long)i * Nx + j) * (Nz + 1) + k;
            w[fw] = w[fw] - f * ProjGrad(g, 2, i, j, k, c, p);
        }
    }
}

// ProjectionGradient3D from the two cell pressures (pc at the face's high cell, pn at its low cell), as ProjGrad.
__device__ __forceinline__ double ProjGradV(const LevelView &g, int a, int i, int j, int k, double pc, double pn)
{
    const int n = a == 0 ? j : (a == 1 ? i : k);
    const double grad = (pc - pn) / Gp(g, a, n - 1);
    const int N = a == 0 ? g.Nx : (a == 1 ? g.Ny : g.Nz);
    if (n != 1 && n != N - 1) return grad;
    const int r = n == 1 ? 0 : N - 1;
    const long long rc = a == 0 ? (long long)i * g.sI + (long long)r * g.sJ + k
                       : (a == 1 ? (long long)r * g.sI + (long long)j * g.sJ + k
                                 : (long long)i * g.sI + (long long)j * g.sJ + r);
    if (!IsDirichlet(g.types[rc])) return grad;
    return n == 1 ? grad * DRF(g, a, 1, -1) : grad * DRF(g, a, N - 2, +1);
}

// The same projection on a 3D grid with Nz even, one thread per cell pair (nb_device.cuh, PairPos) marching along
// i: the pair's u faces and v faces are one aligned 16-byte load and store each (a face outside its loop range or
// behind a wall is stored back unchanged), its two w faces scalars; the pressures of the low neighbours come from
// the pair loads of the previous plane and row and, along k, from the neighbouring lane. The block whose planes end
// at Ny-2 also does the v faces of plane Ny-1 (v's loop runs to Ny-1).
__global__ void __launch_bounds__(kPairThreads) k_pair_project(LevelView g, double *u, double *v, double *w,
                                                               const double *p, double f)
{
    const PairPos P = PairStart(g);
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz, j = P.j;
    const int iEnd = (P.i0 < P.i1 && P.i1 == Ny - 1) ? Ny : P.i1;
    double2 pM = *reinterpret_cast<const double2 *>(p + P.base - P.sI);
    unsigned tM = *reinterpret_cast<const unsigned short *>(g.types + P.base - P.sI);
    int off = 0;
    for (int i = P.i0; i < iEnd; i++, off += P.sI)
    {
        const long long c = P.base + off;
        const double2 pC = *reinterpret_cast<const double2 *>(p + c);
        const unsigned tC = *reinterpret_cast<const unsigned short *>(g.types + c);
        double pKm = __shfl_up_sync(0xffffffffu, pC.y, 1);
        unsigned tKm = __shfl_up_sync(0xffffffffu, tC >> 8, 1);
        if (P.lane == 0)
        {
            pKm = p[c - 1];
            tKm = g.types[c - 1];
        }
        if (P.valid)
        {
            const bool inner = i <= Ny - 2;
            const double pc[2] = {pC.x, pC.y}, pm[2] = {pM.x, pM.y};
            const int tc[2] = {(int)(tC & 0xFFu), (int)(tC >> 8)}, tm[2] = {(int)(tM & 0xFFu), (int)(tM >> 8)};
            // u faces (i, j, k): i in [1, Ny-2], j in [1, Nx-1], k in [1, Nz-2]
            if (inner && j >= 1)
            {
                const long long fu = ((long long)i * (Nx + 1) + j) * Nz + P.k0;
                double2 uu = *reinterpret_cast<double2 *>(u + fu);
                const double2 pJ = *reinterpret_cast<const double2 *>(p + c - P.sJ);
                const unsigned tJ = *reinterpret_cast<const unsigned short *>(g.types + c - P.sJ);
                double ux[2] = {uu.x, uu.y};
                const double pj[2] = {pJ.x, pJ.y};
#pragma unroll
                for (int h = 0; h < 2; h++)
                {
                    const int k = P.k0 + h;
                    if (k < 1 || k > Nz - 2) continue;
                    if (tc[h] == SOLID || (int)((tJ >> (8 * h)) & 0xFFu) == SOLID) continue;
                    ux[h] = ux[h] - f * ProjGradV(g, 0, i, j, k, pc[h], pj[h]);
                }
                *reinterpret_cast<double2 *>(u + fu) = make_double2(ux[0], ux[1]);
            }
            // v faces: i in [1, Ny-1], j in [1, Nx-2], k in [1, Nz-2]
            if (j >= 1 && j <= Nx - 2)
            {
                const long long fv = c; // ((i * Nx + j) * Nz + k): the cell index
                double2 vv = *reinterpret_cast<double2 *>(v + fv);
                double vx[2] = {vv.x, vv.y};
#pragma unroll
                for (int h = 0; h < 2; h++)
                {
                    const int k = P.k0 + h;
                    if (k < 1 || k > Nz - 2) continue;
                    if (tc[h] == SOLID || tm[h] == SOLID) continue;
                    vx[h] = vx[h] - f * ProjGradV(g, 1, i, j, k, pc[h], pm[h]);
                }
                *reinterpret_cast<double2 *>(v + fv) = make_double2(vx[0], vx[1]);
            }
            // w faces: i in [1, Ny-2], j in [1, Nx-2], k in [1, Nz-1]
            if (inner && j >= 1 && j <= Nx - 2)
            {
                const long long fw = ((long long)i * Nx + j) * (Nz + 1) + P.k0;
                const double plow[2] = {pKm, pC.x};
                const int tlow[2] = {(int)tKm, tc[0]};
#pragma unroll
                for (int h = 0; h < 2; h++)
                {
                    const int k = P.k0 + h;
                    if (k < 1 || k > Nz - 1) continue;
                    if (tc[h] == SOLID || tlow[h] == SOLID) continue;
                    w[fw + h] = w[fw + h] - f * ProjGradV(g, 2, i, j, k, pc[h], plow[h]);
                }
            }
        }
        pM = pC;
        tM = tC;
    }
}

void LaunchProject(const LevelView &g, double *u, double *v, double *w, const double *p, double dtOverRho,
                   cudaStream_t st)
{
    if (g.dim == 3 && g.Nz % 2 == 0 && g.Ny >= 3)
    {
        NB_COUNT_LAUNCH();
        k_pair_project<<<PairGrid(g), kPairThreads, 0, st>>>(g, u, v, w, p, dtOverRho);
        return;
    }
    const int kCount = g.dim == 3 ? g.Nz - 1 : 1;
    const int jCount = g.Nx - 1, iCount = g.Ny - 1;
    if (kCount <= 0 || jCount <= 0 || iCount <= 0) return;
    dim3 block(g.dim == 3 ? 32 : 1, g.dim == 3 ? 8 : 256);
    dim3 grid((kCount + block.x - 1) / block.x, (jCount + block.y - 1) / block.y, iCount);
    NB_COUNT_LAUNCH();
    k_project<<<grid, block, 0, st>>>(g, u, v, w, p, dtOverRho);
}

// ---------------------------------------------------------------------------------------------------------------
// compact <-> grid through IDP, and the cell volume (SolveLaplacian, PressureSolver3D.cpp:355-371)
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_gather(LevelView v, const int32_t *idp, const double *grid, double *compact)
{
    const int lane = threadIdx.x & 31, warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int line = warp; line < v.nLines; line += nw)
        for (int f = lane; f < v.lineLen; f += 32)
        {
            int i, j, k;
            long long c;
            LineCell(v, line, f, i, j, k, c);
            const int r = idp[c];
            if (r >= 0) compact[r] = grid[c];
        }
}

__global__ void k_scatter_volume(LevelView v, const int32_t *idp, const double *compact, double *grid, int volume)
{
    const int lane = threadIdx.x & 31, warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int line = warp; line < v.nLines; line += nw)
        for (int f = lane; f < v.lineLen; f += 32)
        {
            int i, j, k;
            long long c;
            LineCell(v, line, f, i, j, k, c);
            const int r = idp[c];
            if (r < 0) continue;
            double vol = 1.0;
            if (volume && v.stretched)
                vol = v.dim == 3 ? Wd(v, 0, j) * Wd(v, 1, i) * Wd(v, 2, k) : Wd(v, 0, j) * Wd(v, 1, i);
            grid[c] = compact[r] * vol;
        }
}

void LaunchGather(const LevelView &v, const int32_t *idp, const double *grid, double *compact, cudaStream_t st)
{
    if (v.nLines <= 0) return;
    NB_COUNT_LAUNCH();
    k_gather<<<LineGrid(v.nLines, 148 * 8), kBlock, 0, st>>>(v, idp, grid, compact);
}

void LaunchScatterVolume(const LevelView &v, const int32_t *idp, const double *compact, double *grid, int volume,
                         cudaStream_t st)
{
    if (v.nLines <= 0) return;
    NB_COUNT_LAUNCH();
    k_scatter_volume<<<LineGrid(v.nLines, 148 * 8), kBlock, 0, st>>>(v, idp, compact, grid, volume);
}

} // namespace nb
