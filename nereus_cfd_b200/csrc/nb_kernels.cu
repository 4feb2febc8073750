// Multigrid and PCG kernels of the B200 pressure solve, on the unit-form operator M = -A/scale (positive
// semi-definite; 5/7-point, face coefficients c_q toward FLUID neighbours, diagonal = sum of fluid faces + Dirichlet
// faces times their ring factor). T = float for the inner solve of the mixed-precision form, double for the plain
// FP64 form. Every vector is zero off the unknowns (interior FLUID cells), which the kernels rely on: they never
// write anywhere else.
//
// Iteration: blocks of 32 x 8 threads tile the (fast, mid) plane of the interior and march along the slow axis
// (nb_device.cuh, TileCell); loads along the fast axis are coalesced 128-byte rows, the neighbours across the tile
// come from L1/L2. A cell's stencil comes from its one-byte code (neighbour-FLUID mask, Dirichlet flag, unknown
// flag), so the common cell reads no neighbour type.
//
// Multigrid (cell-centred, 2:1 coarsening, the hierarchy built in nb_solver.cu):
//   - smoother: red-black Gauss-Seidel, colour (i+j+k)&1, red first before the coarse correction and in reverse
//     order after it, so the V-cycle is a symmetric operator and can precondition CG; a half-sweep launches only
//     the cells of its colour;
//   - restriction: the transpose of the prolongation, summed only from FLUID fine cells into FLUID coarse cells;
//   - prolongation: trilinear, except that a SOLID coarse contributor hands its weight to the child's parent
//     (constant extrapolation across a Neumann wall) and a Dirichlet one keeps its zero; added only at FLUID cells;
//   - coarsest level: symmetric red-black sweeps inside one CTA.
#include "nb_kernels.h"

namespace nb
{

std::atomic<long long> g_launches{0};

static const dim3 kTile(kTileF, kTileM, 1);

#define NB_TILE_LOOP(v)                                                                                            \
    const int fo = blockIdx.x * kTileF + threadIdx.x, mo = blockIdx.y * kTileM + threadIdx.y;                      \
    const int sBeg = blockIdx.z * (v).slowChunk;                                                                   \
    const int sEnd = min(sBeg + (v).slowChunk, (v).slowLen);                                                       \
    for (int s = sBeg; s < sEnd; s++)

// FP64 coefficients of level 0 exactly as the reference forms them (products and divisions only; FaceCoefs3D,
// PressureSolver3D.cpp:47-63; 2D c[] PressureSolver2D.cpp:123-126).
__device__ __forceinline__ void Coefs64(const LevelView &v, int i, int j, int k, double c[6])
{
    if (!v.stretched)
    {
#pragma unroll
        for (int q = 0; q < 6; q++) c[q] = q < (v.dim == 3 ? 6 : 4) ? v.gamma : 0.0;
        return;
    }
    if (v.dim == 2)
    {
        c[0] = Wd(v, 0, j) / Gp(v, 1, i);
        c[1] = Wd(v, 0, j) / Gp(v, 1, i - 1);
        c[2] = Wd(v, 1, i) / Gp(v, 0, j);
        c[3] = Wd(v, 1, i) / Gp(v, 0, j - 1);
        c[4] = c[5] = 0.0;
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

__device__ __forceinline__ double RingFactor64(const LevelView &v, int i, int j, int k, int q)
{
    if (!v.stretched) return 2.0;
    const int a = q < 2 ? 1 : (q < 4 ? 0 : 2);
    const int n = q < 2 ? i : (q < 4 ? j : k);
    const int s = (q & 1) ? -1 : 1;
    return Gp(v, a, s < 0 ? n - 1 : n) / (0.5 * Wd(v, a, n));
}

// Stencil of an unknown cell. kExact: the FP64 tables and the reference's formula (the operator of the FP64 solve's
// CG on level 0); otherwise the level's own (FP32-table) coefficients.
template <typename T, bool kExact>
__device__ __forceinline__ void Stencil(const LevelView &v, int i, int j, int k, long long c, unsigned code, T cq[6],
                                        T &diag)
{
    if (!kExact)
    {
        CodeStencil<T>(v, i, j, k, c, code, cq, diag);
        return;
    }
    double c64[6];
    Coefs64(v, i, j, k, c64);
    double d = 0.0;
#pragma unroll
    for (int q = 0; q < 6; q++)
        if (code >> q & 1u) d += c64[q];
    if (code & CODE_DIRICHLET)
    {
        const int nq = v.dim == 3 ? 6 : 4;
        for (int q = 0; q < nq; q++)
        {
            const int t = v.types[c + NbrOffset(v, q)];
            if (IsDirichlet(t))
            {
                const int ni = i + (q == 0) - (q == 1), nj = j + (q == 2) - (q == 3), nk = k + (q == 4) - (q == 5);
                d += OnRing(v, ni, nj, nk) ? c64[q] * RingFactor64(v, i, j, k, q) : c64[q];
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 6; q++) cq[q] = (T)c64[q];
    diag = (T)d;
}

// sum over the FLUID neighbours of c_q x_q
template <typename T>
__device__ __forceinline__ T OffSum(const LevelView &v, long long c, unsigned code, const T cq[6], const T *x)
{
    T s = (T)0;
    if (code & 1u) s += cq[0] * x[c + v.sI];
    if (code & 2u) s += cq[1] * x[c - v.sI];
    if (code & 4u) s += cq[2] * x[c + v.sJ];
    if (code & 8u) s += cq[3] * x[c - v.sJ];
    if (code & 16u) s += cq[4] * x[c + 1];
    if (code & 32u) s += cq[5] * x[c - 1];
    return s;
}

// the six neighbours of an interior cell, loaded unconditionally (all in bounds; 2D reads its j neighbours twice)
template <typename T>
__device__ __forceinline__ void LoadNbrs(const LevelView &v, long long c, const T *x, T xn[6])
{
    xn[0] = x[c + v.sI];
    xn[1] = x[c - v.sI];
    xn[2] = x[c + v.sJ];
    xn[3] = x[c - v.sJ];
    xn[4] = x[c + 1];
    xn[5] = x[c - 1];
}

// sum over the FLUID neighbours (code bits 0-5) of c_q x_q
template <typename T> __device__ __forceinline__ T MaskedSum(unsigned code, const T cq[6], const T xn[6])
{
    T s = (T)0;
#pragma unroll
    for (int q = 0; q < 6; q++) s += ((code >> q) & 1u) ? cq[q] * xn[q] : (T)0;
    return s;
}

// ---------------------------------------------------------------------------------------------------------------
// per-level cell codes and coarse cell types
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_build_codes(LevelView v, uint8_t *code)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < v.cells;
         c += (long long)gridDim.x * blockDim.x)
    {
        const int k = (int)(c % v.Nz);
        const long long r = c / v.Nz;
        const int j = (int)(r % v.Nx), i = (int)(r / v.Nx);
        const bool interior = i > 0 && i < v.Ny - 1 && j > 0 && j < v.Nx - 1 &&
                              (v.dim == 2 || (k > 0 && k < v.Nz - 1));
        if (!interior || v.types[c] != FLUID) { code[c] = 0; continue; }
        unsigned m = CODE_UNKNOWN;
        const int nq = v.dim == 3 ? 6 : 4;
        for (int q = 0; q < nq; q++)
        {
            const int t = v.types[c + NbrOffset(v, q)];
            if (t == FLUID) m |= 1u << q;
            else if (IsDirichlet(t)) m |= CODE_DIRICHLET;
        }
        code[c] = (uint8_t)m;
    }
}

void LaunchBuildCodes(const LevelView &v, uint8_t *code, cudaStream_t st)
{
    int blocks = (int)((v.cells + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    NB_COUNT_LAUNCH();
    k_build_codes<<<blocks, 256, 0, st>>>(v, code);
}

// An interior coarse cell is Dirichlet (EMPTY) if any child is, else FLUID if any child is, else SOLID (Neumann); a
// coarse ring cell on one face is Dirichlet if any of its ring children is Dirichlet or FLUID, else SOLID; ring
// edges and corners are SOLID.
__global__ void k_coarsen_types(LevelView f, LevelView cv, uint8_t *ct)
{
    const long long cells = cv.cells;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells;
         c += (long long)gridDim.x * blockDim.x)
    {
        const int K = (int)(c % cv.Nz);
        const long long r = c / cv.Nz;
        const int J = (int)(r % cv.Nx), I = (int)(r / cv.Nx);
        const bool rI = I == 0 || I == cv.Ny - 1, rJ = J == 0 || J == cv.Nx - 1;
        const bool rK = cv.dim == 3 && (K == 0 || K == cv.Nz - 1);
        const int codim = (int)rI + (int)rJ + (int)rK;
        if (codim >= 2) { ct[c] = SOLID; continue; }
        int ia[2], ja[2], ka[2], ni = 0, nj = 0, nk = 0;
        auto kids = [](int C, int Nc, int Nf, int *out, int &cnt) {
            if (C == 0) { out[0] = 0; cnt = 1; return; }
            if (C == Nc - 1) { out[0] = Nf - 1; cnt = 1; return; }
            out[0] = 2 * C - 1;
            cnt = 1;
            if (2 * C <= Nf - 2) out[cnt++] = 2 * C;
        };
        kids(I, cv.Ny, f.Ny, ia, ni);
        if (f.xr)
        {
            const int x = f.xr[J];
            ja[0] = x & 0x7FFF;
            ja[1] = ja[0] + 1;
            nj = (x >> 15) & 1 ? 2 : 1;
        }
        else kids(J, cv.Nx, f.Nx, ja, nj);
        if (cv.dim == 3) kids(K, cv.Nz, f.Nz, ka, nk);
        else { ka[0] = 0; nk = 1; }
        bool anyDir = false, anyFluid = false;
        for (int a = 0; a < ni; a++)
            for (int b = 0; b < nj; b++)
                for (int d = 0; d < nk; d++)
                {
                    const int t = f.types[(long long)ia[a] * f.sI + (long long)ja[b] * f.sJ + ka[d]];
                    anyDir |= IsDirichlet(t);
                    anyFluid |= (t == FLUID);
                }
        if (codim == 1) ct[c] = (anyDir || anyFluid) ? EMPTY : SOLID;
        else ct[c] = anyDir ? EMPTY : (anyFluid ? FLUID : SOLID);
    }
}

void LaunchCoarsenTypes(const LevelView &fine, const LevelView &coarse, uint8_t *coarseTypes, cudaStream_t st)
{
    int blocks = (int)((coarse.cells + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    NB_COUNT_LAUNCH();
    k_coarsen_types<<<blocks, 256, 0, st>>>(fine, coarse, coarseTypes);
}

// ---------------------------------------------------------------------------------------------------------------
// smoother: one colour of a red-black sweep. kFirst: the red pass from a zero iterate (e = r / diag; the black
// values that follow never read the old black ones, so nothing else needs clearing).
// ---------------------------------------------------------------------------------------------------------------
template <typename T, bool kFirst>
__global__ void __launch_bounds__(256) k_smooth(LevelView v, const T *__restrict__ r, T *e, int colour)
{
    NB_TILE_LOOP(v)
    {
        int i, j, k;
        long long c;
        if (!TileCellColour(v, fo, mo, s, colour, i, j, k, c)) continue;
        // every load of the cell is issued before anything depends on one of them
        const unsigned code = v.code[c];
        const T rc = r[c];
        T xn[6];
        if (!kFirst) LoadNbrs<T>(v, c, e, xn);
        if (!(code & CODE_UNKNOWN)) continue;
        T cq[6], diag;
        CodeStencil<T>(v, i, j, k, c, code, cq, diag);
        const T rhs = kFirst ? rc : rc + MaskedSum<T>(code, cq, xn);
        e[c] = diag != (T)0 ? rhs / diag : (T)0;
    }
}

// Stencil launches with no reduction take one slow-axis step per block: many blocks, many warps per SM.
static inline LevelView OnePlane(const LevelView &v)
{
    LevelView o = v;
    o.slowChunk = 1;
    return o;
}

template <typename T> void LaunchSmoothFirst(const LevelView &v, const T *r, T *e, cudaStream_t st)
{
    if (v.fastLen <= 0 || v.midLen <= 0) return;
    const LevelView o = OnePlane(v);
    NB_COUNT_LAUNCH();
    k_smooth<T, true><<<TileGrid(o, true), kTile, 0, st>>>(o, r, e, 0);
}

template <typename T> void LaunchSmooth(const LevelView &v, const T *r, T *e, int colour, cudaStream_t st)
{
    if (v.fastLen <= 0 || v.midLen <= 0) return;
    const LevelView o = OnePlane(v);
    NB_COUNT_LAUNCH();
    k_smooth<T, false><<<TileGrid(o, true), kTile, 0, st>>>(o, r, e, colour);
}

// res = r - M e
template <typename T>
__global__ void __launch_bounds__(256) k_level_residual(LevelView v, const T *__restrict__ r, const T *__restrict__ e,
                                                        T *__restrict__ res)
{
    NB_TILE_LOOP(v)
    {
        int i, j, k;
        long long c;
        if (!TileCell(v, fo, mo, s, i, j, k, c)) continue;
        const unsigned code = v.code[c];
        const T rc = r[c], ec = e[c];
        T xn[6];
        LoadNbrs<T>(v, c, e, xn);
        if (!(code & CODE_UNKNOWN)) continue;
        T cq[6], diag;
        CodeStencil<T>(v, i, j, k, c, code, cq, diag);
        res[c] = rc - (diag * ec - MaskedSum<T>(code, cq, xn));
    }
}

template <typename T> void LaunchLevelResidual(const LevelView &v, const T *r, const T *e, T *res, cudaStream_t st)
{
    if (v.fastLen <= 0 || v.midLen <= 0) return;
    const LevelView o = OnePlane(v);
    NB_COUNT_LAUNCH();
    k_level_residual<T><<<TileGrid(o), kTile, 0, st>>>(o, r, e, res);
}

// ---------------------------------------------------------------------------------------------------------------
// transfers
// ---------------------------------------------------------------------------------------------------------------

// Weight the prolongation moves onto coarse cell (I,J,K) from the SOLID contributors of its child on side
// (si, sj, sk): the sum of the trilinear weights of those contributors.
template <typename T>
__device__ __forceinline__ T SolidWeight(const LevelView &cv, int I, int J, int K, int si, int sj, int sk)
{
    const T wv[2] = {(T)0.75, (T)0.25};
    const long long parent = (long long)I * cv.sI + (long long)J * cv.sJ + K;
    T extra = (T)0;
    const int nk = cv.dim == 3 ? 2 : 1;
    for (int di = 0; di < 2; di++)
        for (int dj = 0; dj < 2; dj++)
            for (int dk = 0; dk < nk; dk++)
            {
                if (!(di | dj | dk)) continue;
                const long long cc = parent + (long long)(di * si) * cv.sI + (long long)(dj * sj) * cv.sJ + dk * sk;
                if (cv.types[cc] == SOLID) extra += wv[di] * wv[dj] * (cv.dim == 3 ? wv[dk] : (T)1);
            }
    return extra;
}

template <typename T>
__global__ void __launch_bounds__(256) k_restrict(LevelView fv, LevelView cv, const T *__restrict__ res,
                                                  T *__restrict__ rc)
{
    NB_TILE_LOOP(cv)
    {
        int I, J, K;
        long long c;
        if (!TileCell(cv, fo, mo, s, I, J, K, c)) continue;
        if (!(cv.code[c] & CODE_UNKNOWN)) continue;
        T acc = (T)0;
        const T wt[4] = {(T)0.25, (T)0.75, (T)0.75, (T)0.25};
        for (int di = 0; di < 4; di++)
        {
            const int a = 2 * I - 2 + di;
            if (a > fv.Ny - 1) continue;
            for (int dj = 0; dj < 4; dj++)
            {
                const int b = 2 * J - 2 + dj;
                if (b > fv.Nx - 1) continue;
                const long long rowBase = (long long)a * fv.sI + (long long)b * fv.sJ;
                const T wij = wt[di] * wt[dj];
                if (fv.dim == 3)
                {
                    T t = (T)0;
#pragma unroll
                    for (int dk = 0; dk < 4; dk++)
                    {
                        const int d = 2 * K - 2 + dk;
                        if (d <= fv.Nz - 1) t += wt[dk] * res[rowBase + d];
                    }
                    acc += wij * t;
                }
                else
                    acc += wij * res[rowBase];
            }
        }
        // the children of (I, J, K) also carry the weight the prolongation moved off their SOLID coarse contributors
        const int nz = fv.dim == 3 ? 2 : 1;
        for (int ci = 0; ci < 2; ci++)
            for (int cj = 0; cj < 2; cj++)
                for (int ck = 0; ck < nz; ck++)
                {
                    const int a = 2 * I - 1 + ci, b = 2 * J - 1 + cj, d = fv.dim == 3 ? 2 * K - 1 + ck : 0;
                    if (a > fv.Ny - 2 || b > fv.Nx - 2 || (fv.dim == 3 && d > fv.Nz - 2)) continue;
                    const T extra = SolidWeight<T>(cv, I, J, K, ci ? 1 : -1, cj ? 1 : -1, ck ? 1 : -1);
                    if (extra != (T)0) acc += extra * res[(long long)a * fv.sI + (long long)b * fv.sJ + d];
                }
        rc[c] = acc;
    }
}

// The same two operators where the coarsening keeps some x cells whole (3D, LevelView::xp / xr): along x a fine cell
// gives its parent 1 (a parent of one child) or 3/4 and the neighbouring coarse cell on its side 1/4; along y and z
// 3/4 and 1/4 as above. SolidWeightX: the weight the prolongation moves onto the parent of fine cell (., b, .) from
// its SOLID contributors (si, sk: the directions of its other contributors along i and k).
template <typename T>
__device__ __forceinline__ T SolidWeightX(const LevelView &fv, const LevelView &cv, int I, int J, int K, int si, int b,
                                          int sk)
{
    const int x = fv.xp[b];
    const bool one = XpSingle(x);
    const int J2 = XpOther(x);
    const T wv[2] = {(T)0.75, (T)0.25};
    const T wj[2] = {one ? (T)1 : (T)0.75, (T)0.25};
    T extra = (T)0;
    for (int di = 0; di < 2; di++)
        for (int dj = 0; dj < (one ? 1 : 2); dj++)
            for (int dk = 0; dk < 2; dk++)
            {
                if (!(di | dj | dk)) continue;
                const long long cc = (long long)(I + di * si) * cv.sI + (long long)(dj ? J2 : J) * cv.sJ + K + dk * sk;
                if (cv.types[cc] == SOLID) extra += wv[di] * wj[dj] * wv[dk];
            }
    return extra;
}

template <typename T>
__global__ void __launch_bounds__(256) k_restrict_x(LevelView fv, LevelView cv, const T *__restrict__ res,
                                                    T *__restrict__ rc)
{
    NB_TILE_LOOP(cv)
    {
        int I, J, K;
        long long c;
        if (!TileCell(cv, fo, mo, s, I, J, K, c)) continue;
        if (!(cv.code[c] & CODE_UNKNOWN)) continue;
        int bq[4];
        T wq[4];
        bool two;
        XrTaps<T>(fv.xr[J], bq, wq, two);
        const T wt[4] = {(T)0.25, (T)0.75, (T)0.75, (T)0.25};
        T acc = (T)0;
        for (int di = 0; di < 4; di++)
        {
            const int a = 2 * I - 2 + di;
            if (a > fv.Ny - 1) continue;
            for (int dj = 0; dj < 4; dj++)
            {
                if (wq[dj] == (T)0) continue;
                const long long rowBase = (long long)a * fv.sI + (long long)bq[dj] * fv.sJ;
                T t = (T)0;
#pragma unroll
                for (int dk = 0; dk < 4; dk++)
                {
                    const int d = 2 * K - 2 + dk;
                    if (d <= fv.Nz - 1) t += wt[dk] * res[rowBase + d];
                }
                acc += (wt[di] * wq[dj]) * t;
            }
        }
        for (int ci = 0; ci < 2; ci++)
            for (int cj = 0; cj < (two ? 2 : 1); cj++)
                for (int ck = 0; ck < 2; ck++)
                {
                    const int a = 2 * I - 1 + ci, b = bq[1] + cj, d = 2 * K - 1 + ck;
                    if (a > fv.Ny - 2 || d > fv.Nz - 2) continue;
                    const T extra = SolidWeightX<T>(fv, cv, I, J, K, ci ? 1 : -1, b, ck ? 1 : -1);
                    if (extra != (T)0) acc += extra * res[(long long)a * fv.sI + (long long)b * fv.sJ + d];
                }
        rc[c] = acc;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_prolong_x(LevelView fv, LevelView cv, const T *__restrict__ ec, T *ef)
{
    NB_TILE_LOOP(fv)
    {
        int a, b, d;
        long long c;
        if (!TileCell(fv, fo, mo, s, a, b, d, c)) continue;
        if (!(fv.code[c] & CODE_UNKNOWN)) continue;
        const int A = (a + 1) >> 1, D = (d + 1) >> 1;
        const int si = (a & 1) ? -1 : 1, sk = (d & 1) ? -1 : 1;
        const int x = fv.xp[b];
        const int B = XpParent(x), B2 = XpOther(x);
        const bool one = XpSingle(x);
        const T wv[2] = {(T)0.75, (T)0.25};
        const T wj[2] = {one ? (T)1 : (T)0.75, (T)0.25};
        const long long parent = (long long)A * cv.sI + (long long)B * cv.sJ + D;
        T acc = (T)0, extra = (T)0;
        for (int di = 0; di < 2; di++)
            for (int dj = 0; dj < (one ? 1 : 2); dj++)
                for (int dk = 0; dk < 2; dk++)
                {
                    const long long cc = (long long)(A + di * si) * cv.sI + (long long)(dj ? B2 : B) * cv.sJ + D + dk * sk;
                    const T w = wv[di] * wj[dj] * wv[dk];
                    if ((di | dj | dk) && cv.types[cc] == SOLID) extra += w; // Neumann: the parent's value
                    else acc += w * ec[cc];
                }
        ef[c] += acc + extra * ec[parent];
    }
}

template <typename T>
void LaunchRestrict(const LevelView &fine, const LevelView &coarse, const T *resFine, T *rCoarse, cudaStream_t st)
{
    if (coarse.fastLen <= 0 || coarse.midLen <= 0) return;
    const LevelView o = OnePlane(coarse);
    NB_COUNT_LAUNCH();
    if (fine.xr) k_restrict_x<T><<<TileGrid(o), kTile, 0, st>>>(fine, o, resFine, rCoarse);
    else k_restrict<T><<<TileGrid(o), kTile, 0, st>>>(fine, o, resFine, rCoarse);
}

template <typename T>
__global__ void __launch_bounds__(256) k_prolong(LevelView fv, LevelView cv, const T *__restrict__ ec, T *ef)
{
    NB_TILE_LOOP(fv)
    {
        int a, b, d;
        long long c;
        if (!TileCell(fv, fo, mo, s, a, b, d, c)) continue;
        if (!(fv.code[c] & CODE_UNKNOWN)) continue;
        const int A = (a + 1) >> 1, B = (b + 1) >> 1;
        const int D = fv.dim == 3 ? (d + 1) >> 1 : 0;
        const int si = (a & 1) ? -1 : 1, sj = (b & 1) ? -1 : 1, sk = (d & 1) ? -1 : 1;
        const T wv[2] = {(T)0.75, (T)0.25};
        const long long parent = (long long)A * cv.sI + (long long)B * cv.sJ + D;
        T acc = (T)0, extra = (T)0;
        const int nk = fv.dim == 3 ? 2 : 1;
        for (int di = 0; di < 2; di++)
            for (int dj = 0; dj < 2; dj++)
                for (int dk = 0; dk < nk; dk++)
                {
                    const long long cc = parent + (long long)(di * si) * cv.sI + (long long)(dj * sj) * cv.sJ + dk * sk;
                    const T w = wv[di] * wv[dj] * (fv.dim == 3 ? wv[dk] : (T)1);
                    if ((di | dj | dk) && cv.types[cc] == SOLID) extra += w; // Neumann: the parent's value
                    else acc += w * ec[cc];
                }
        ef[c] += acc + extra * ec[parent];
    }
}

template <typename T>
void LaunchProlong(const LevelView &fine, const LevelView &coarse, const T *eCoarse, T *eFine, cudaStream_t st)
{
    if (fine.fastLen <= 0 || fine.midLen <= 0) return;
    const LevelView o = OnePlane(fine);
    NB_COUNT_LAUNCH();
    if (fine.xp) k_prolong_x<T><<<TileGrid(o), kTile, 0, st>>>(o, coarse, eCoarse, eFine);
    else k_prolong<T><<<TileGrid(o), kTile, 0, st>>>(o, coarse, eCoarse, eFine);
}

// ---------------------------------------------------------------------------------------------------------------
// coarsest level: `sweeps` forward red-black pairs then as many backward black-red pairs, from zero, in one CTA
// ---------------------------------------------------------------------------------------------------------------
template <typename T>
__device__ void CoarseHalf(const LevelView &v, const T *r, T *e, int colour, int first)
{
    for (long long c = threadIdx.x; c < v.cells; c += blockDim.x)
    {
        const unsigned code = v.code[c];
        if (!(code & CODE_UNKNOWN)) continue;
        const int k = (int)(c % v.Nz);
        const long long rr = c / v.Nz;
        const int j = (int)(rr % v.Nx), i = (int)(rr / v.Nx);
        const int col = (i + j + k) & 1;
        if (col != colour) continue;
        T cq[6], diag;
        CodeStencil<T>(v, i, j, k, c, code, cq, diag);
        const T rhs = first ? r[c] : r[c] + OffSum<T>(v, c, code, cq, e);
        e[c] = diag != (T)0 ? rhs / diag : (T)0;
    }
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(1024) k_coarse(LevelView v, const T *r, T *e, int sweeps)
{
    CoarseHalf<T>(v, r, e, 0, 1);
    CoarseHalf<T>(v, r, e, 1, 0);
    for (int s = 1; s < sweeps; s++)
    {
        CoarseHalf<T>(v, r, e, 0, 0);
        CoarseHalf<T>(v, r, e, 1, 0);
    }
    for (int s = 0; s < sweeps; s++)
    {
        CoarseHalf<T>(v, r, e, 1, 0);
        CoarseHalf<T>(v, r, e, 0, 0);
    }
}

template <typename T> void LaunchCoarseSolve(const LevelView &v, const T *r, T *e, int sweeps, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_coarse<T><<<1, 1024, 0, st>>>(v, r, e, sweeps < 1 ? 1 : sweeps);
}

// ---------------------------------------------------------------------------------------------------------------
// PCG
// ---------------------------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_dot(LevelView v, const T *__restrict__ r, const T *__restrict__ z, Reducer R,
                                             const int *it, int baseEven, int baseOdd)
{
    const int base = (*it & 1) ? baseOdd : baseEven;
    double acc[3] = {0.0, 0.0, 0.0};
    NB_TILE_LOOP(v)
    {
        int i, j, k;
        long long c;
        if (!TileCell(v, fo, mo, s, i, j, k, c)) continue;
        const double rv = (double)r[c], zv = (double)z[c];
        acc[0] += rv * zv;
        acc[1] += zv;
        acc[2] += rv;
    }
    GridReduce<3>(R, acc, base);
}

template <typename T>
void LaunchDot(const LevelView &v, const T *r, const T *z, const Reducer &R, const int *it, int baseEven, int baseOdd,
               cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_dot<T><<<TileGrid(v), kTile, 0, st>>>(v, r, z, R, it, baseEven, baseOdd);
}

// n (the unknowns) is read from S[slotN] on the device, so a captured iteration outlives a change of the layout
// that keeps the hierarchy's shape
__device__ __forceinline__ double RzEff(const double *S, int base, double n, int singular)
{
    return singular ? S[base] - (S[base + 1] / n) * S[base + 2] : S[base];
}

// p_new = (z - mean) + beta p_old, q = M p_new, sum p_new.q. The neighbours' p_new are formed from their z and
// p_old, so p_old and p_new are different arrays. Every load of a cell is issued before any depends on another.
template <typename T, bool kExact>
__global__ void __launch_bounds__(256) k_update_p_apply(LevelView v, const T *__restrict__ z, T *p0, T *p1,
                                                        T *__restrict__ q, Reducer R, const double *S, const int *it,
                                                        int baseEven, int baseOdd, int slotN, int singular, int slotPQ)
{
    const int iter = *it, par = iter & 1;
    const T *__restrict__ pIn = par ? p1 : p0;
    T *__restrict__ pOut = par ? p0 : p1;
    const int baseNew = par ? baseOdd : baseEven, baseOld = par ? baseEven : baseOdd;
    const double n = S[slotN];
    const double beta = iter == 0 ? 0.0 : RzEff(S, baseNew, n, singular) / RzEff(S, baseOld, n, singular);
    const T b = (T)beta;
    const T mean = singular ? (T)(S[baseNew + 1] / n) : (T)0;
    double acc[1] = {0.0};
    NB_TILE_LOOP(v)
    {
        int i, j, k;
        long long c;
        if (!TileCell(v, fo, mo, s, i, j, k, c)) continue;
        const unsigned code = v.code[c];
        const long long o[6] = {v.sI, -v.sI, v.sJ, -v.sJ, 1, -1};
        T zn[6], pn[6];
#pragma unroll
        for (int qq = 0; qq < 6; qq++)
        {
            zn[qq] = z[c + o[qq]];
            pn[qq] = pIn[c + o[qq]];
        }
        const T zc = z[c], pcOld = pIn[c];
        if (!(code & CODE_UNKNOWN)) continue;
        T cq[6], diag;
        Stencil<T, kExact>(v, i, j, k, c, code, cq, diag);
        const T pc = (zc - mean) + b * pcOld;
        T sum = diag * pc;
#pragma unroll
        for (int qq = 0; qq < 6; qq++)
        {
            T pnew = (zn[qq] - mean) + b * pn[qq];
            if (singular)
            {
                const int ni = i + (qq == 0) - (qq == 1), nj = j + (qq == 2) - (qq == 3), nk = k + (qq == 4) - (qq == 5);
                if (OnRing(v, ni, nj, nk)) pnew = (T)0;
            }
            sum -= ((code >> qq) & 1u) ? cq[qq] * pnew : (T)0;
        }
        pOut[c] = pc;
        q[c] = sum;
        acc[0] += (double)pc * (double)sum;
    }
    GridReduce<1>(R, acc, slotPQ);
}

template <typename T>
void LaunchUpdatePApply(const LevelView &v, const T *z, T *p0, T *p1, T *q, const Reducer &R, const double *S,
                        const int *it, int baseEven, int baseOdd, int slotN, int singular, int slotPQ, int exact,
                        cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    if (exact)
        k_update_p_apply<T, true><<<TileGrid(v), kTile, 0, st>>>(v, z, p0, p1, q, R, S, it, baseEven, baseOdd, slotN,
                                                                 singular, slotPQ);
    else
        k_update_p_apply<T, false><<<TileGrid(v), kTile, 0, st>>>(v, z, p0, p1, q, R, S, it, baseEven, baseOdd, slotN,
                                                                  singular, slotPQ);
}

// alpha = rz/pq; x += alpha p_new; r -= alpha q; sum r.r. The last block advances the iteration counter.
template <typename T>
__global__ void __launch_bounds__(256) k_update_xr(LevelView v, T *__restrict__ x, T *__restrict__ r, const T *p0,
                                                   const T *p1, const T *__restrict__ q, Reducer R, const double *S,
                                                   int *it, int baseEven, int baseOdd, int slotN, int singular,
                                                   int slotPQ, int slotRR)
{
    const int par = *it & 1;
    const T *__restrict__ p = par ? p0 : p1;
    const int base = par ? baseOdd : baseEven;
    const double alpha = RzEff(S, base, S[slotN], singular) / S[slotPQ];
    const T a = (T)alpha;
    double acc[1] = {0.0};
    NB_TILE_LOOP(v)
    {
        int i, j, k;
        long long c;
        if (!TileCell(v, fo, mo, s, i, j, k, c)) continue;
        const T pv = p[c], qv = q[c], xv = x[c], rv = r[c];
        x[c] = xv + a * pv;
        const T rn = rv - a * qv;
        r[c] = rn;
        acc[0] += (double)rn * (double)rn;
    }
    GridReduce<1>(R, acc, slotRR, 0, it);
}

template <typename T>
void LaunchUpdateXR(const LevelView &v, T *x, T *r, const T *p0, const T *p1, const T *q, const Reducer &R,
                    const double *S, int *it, int baseEven, int baseOdd, int slotN, int singular, int slotPQ, int slotRR,
                    cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_update_xr<T><<<TileGrid(v), kTile, 0, st>>>(v, x, r, p0, p1, q, R, S, it, baseEven, baseOdd, slotN, singular,
                                                  slotPQ, slotRR);
}

template <typename Tin, typename Tout>
__global__ void __launch_bounds__(256) k_scale_copy(LevelView v, const Tin *x, Tout *y, double sc)
{
    NB_TILE_LOOP(v)
    {
        int i, j, k;
        long long c;
        if (!TileCell(v, fo, mo, s, i, j, k, c)) continue;
        if (!(v.code[c] & CODE_UNKNOWN)) continue;
        y[c] = (Tout)((double)x[c] * sc);
    }
}

template <typename Tin, typename Tout>
void LaunchScaleCopy(const LevelView &v, const Tin *x, Tout *y, double s, cudaStream_t st)
{
    if (v.fastLen <= 0 || v.midLen <= 0) return;
    NB_COUNT_LAUNCH();
    k_scale_copy<Tin, Tout><<<TileGrid(v), kTile, 0, st>>>(v, x, y, s);
}

// (count of unknowns, count of unknowns whose row reaches a Dirichlet neighbour or a FLUID ring cell): the system
// size and, when the second is 0, the singular (all-Neumann) case (AssembleSystem's `dirichlet`,
// PressureSolver3D.cpp:128-178).
__global__ void __launch_bounds__(256) k_count_unknowns(LevelView v, Reducer R, int slot)
{
    double acc[2] = {0.0, 0.0};
    NB_TILE_LOOP(v)
    {
        int i, j, k;
        long long c;
        if (!TileCell(v, fo, mo, s, i, j, k, c)) continue;
        const unsigned code = v.code[c];
        if (!(code & CODE_UNKNOWN)) continue;
        acc[0] += 1.0;
        bool dir = (code & CODE_DIRICHLET) != 0;
        const int nq = v.dim == 3 ? 6 : 4;
        for (int q = 0; q < nq && !dir; q++)
            if ((code >> q) & 1u)
                dir = OnRing(v, i + (q == 0) - (q == 1), j + (q == 2) - (q == 3), k + (q == 4) - (q == 5));
        if (dir) acc[1] += 1.0;
    }
    GridReduce<2>(R, acc, slot);
}

void LaunchCountUnknowns(const LevelView &v, const Reducer &R, int slot, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_count_unknowns<<<TileGrid(v), kTile, 0, st>>>(v, R, slot);
}

// r = sfac * b over the whole level and (sum b^2, sum b): the FP64 residual b - A x of a zero iterate. b is zero off
// the unknowns, so the sums over all cells are the sums over the unknowns.
template <typename T>
__global__ void __launch_bounds__(256) k_scale_sum(long long cells, const double *__restrict__ b, T *__restrict__ r,
                                                   double sfac, Reducer R, int slot)
{
    double acc[2] = {0.0, 0.0};
    const long long n2 = cells >> 1, stride = (long long)gridDim.x * blockDim.x;
    const double2 *b2 = reinterpret_cast<const double2 *>(b);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n2; t += stride)
    {
        const double2 x = b2[t];
        r[2 * t] = (T)(x.x * sfac);
        r[2 * t + 1] = (T)(x.y * sfac);
        acc[0] += x.x * x.x + x.y * x.y;
        acc[1] += x.x + x.y;
    }
    for (long long t = 2 * n2 + blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cells; t += stride)
    {
        r[t] = (T)(b[t] * sfac);
        acc[0] += b[t] * b[t];
        acc[1] += b[t];
    }
    GridReduce<2>(R, acc, slot);
}

template <typename T>
void LaunchScaleSum(long long cells, const double *b, T *r, double sfac, const Reducer &R, int slot, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_scale_sum<T><<<148 * 8, 256, 0, st>>>(cells, b, r, sfac, R, slot);
}
template void LaunchScaleSum<float>(long long, const double *, float *, double, const Reducer &, int, cudaStream_t);
template void LaunchScaleSum<double>(long long, const double *, double *, double, const Reducer &, int, cudaStream_t);

// ---- instantiations ----
#define NB_INST(T)                                                                                                 \
    template void LaunchSmoothFirst<T>(const LevelView &, const T *, T *, cudaStream_t);                           \
    template void LaunchSmooth<T>(const LevelView &, const T *, T *, int, cudaStream_t);                           \
    template void LaunchLevelResidual<T>(const LevelView &, const T *, const T *, T *, cudaStream_t);              \
    template void LaunchRestrict<T>(const LevelView &, const LevelView &, const T *, T *, cudaStream_t);           \
    template void LaunchProlong<T>(const LevelView &, const LevelView &, const T *, T *, cudaStream_t);            \
    template void LaunchCoarseSolve<T>(const LevelView &, const T *, T *, int, cudaStream_t);                      \
    template void LaunchDot<T>(const LevelView &, const T *, const T *, const Reducer &, const int *, int, int,     \
                               cudaStream_t);                                                                      \
    template void LaunchUpdatePApply<T>(const LevelView &, const T *, T *, T *, T *, const Reducer &,              \
                                        const double *, const int *, int, int, int, int, int, int, cudaStream_t);  \
    template void LaunchUpdateXR<T>(const LevelView &, T *, T *, const T *, const T *, const T *, const Reducer &, \
                                    const double *, int *, int, int, int, int, int, int, cudaStream_t);
NB_INST(float)
NB_INST(double)
template void LaunchScaleCopy<double, float>(const LevelView &, const double *, float *, double, cudaStream_t);
template void LaunchScaleCopy<double, double>(const LevelView &, const double *, double *, double, cudaStream_t);
template void LaunchScaleCopy<float, double>(const LevelView &, const float *, double *, double, cudaStream_t);

} // namespace nb
