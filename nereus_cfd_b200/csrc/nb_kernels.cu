// Multigrid and PCG kernels of the B200 pressure solve, on the unit-form operator M = -A/scale (positive
// semi-definite; 5/7-point, face coefficients c_q toward FLUID neighbours, diagonal = sum of fluid faces + Dirichlet
// faces times their ring factor). T = float for the inner solve of the mixed-precision form, double for the plain
// FP64 form. Every vector is zero off the unknowns (interior FLUID cells), which the kernels rely on: they never
// write anywhere else.
//
// Multigrid (cell-centred, 2:1 coarsening, the hierarchy built in nb_solver.cu):
//   - smoother: red-black Gauss-Seidel, colour (i+j+k)&1, red first before the coarse correction and in reverse
//     order after it, so the V-cycle is a symmetric operator and can precondition CG;
//   - restriction: the transpose of the prolongation (weights 1/4, 3/4, 3/4, 1/4 per axis over the 4-wide fine
//     window), summed only from FLUID fine cells into FLUID coarse cells;
//   - prolongation: trilinear (3/4 parent, 1/4 the neighbour on the child's side per axis), added only at FLUID
//     fine cells; coarse cells that are not FLUID hold zero;
//   - coarsest level: symmetric red-black sweeps inside one CTA.
#include "nb_kernels.h"

namespace nb
{

std::atomic<long long> g_launches{0};

// FP64 coefficients of level 0 exactly as the reference forms them (products and divisions only; FaceCoefs3D,
// PressureSolver3D.cpp:47-63; 2D c[] PressureSolver2D.cpp:123-126).
__device__ __forceinline__ void Coefs64(const LevelView &v, int i, int j, int k, double c[6])
{
    if (v.dim == 2)
    {
        if (!v.stretched) { c[0] = c[1] = c[2] = c[3] = v.gamma; c[4] = c[5] = 0.0; return; }
        c[0] = Wd(v, 0, j) / Gp(v, 1, i);
        c[1] = Wd(v, 0, j) / Gp(v, 1, i - 1);
        c[2] = Wd(v, 1, i) / Gp(v, 0, j);
        c[3] = Wd(v, 1, i) / Gp(v, 0, j - 1);
        c[4] = c[5] = 0.0;
        return;
    }
    if (!v.stretched)
    {
#pragma unroll
        for (int q = 0; q < 6; q++) c[q] = v.gamma;
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

// Stencil of FLUID cell c: off-diagonal magnitudes cq, diagonal, and which neighbours are FLUID.
// kExact: the FP64 tables and the reference's formula (level 0 of the FP64 solve); otherwise LevelStencil.
template <typename T, bool kExact>
__device__ __forceinline__ void Stencil(const LevelView &v, int i, int j, int k, long long c, T cq[6], T &diag,
                                        unsigned &mask)
{
    if (!kExact)
    {
        LevelStencil<T>(v, i, j, k, c, cq, diag, mask);
        return;
    }
    double c64[6];
    Coefs64(v, i, j, k, c64);
    const int nq = v.dim == 3 ? 6 : 4;
    double d = 0.0;
    unsigned m = 0;
    for (int q = 0; q < nq; q++)
    {
        const int t = v.types[c + NbrOffset(v, q)];
        if (t == FLUID) { d += c64[q]; m |= 1u << q; }
    }
    for (int q = 0; q < nq; q++)
    {
        const int t = v.types[c + NbrOffset(v, q)];
        if (IsDirichlet(t))
        {
            const int ni = i + (q == 0) - (q == 1), nj = j + (q == 2) - (q == 3), nk = k + (q == 4) - (q == 5);
            d += OnRing(v, ni, nj, nk) ? c64[q] * RingFactor64(v, i, j, k, q) : c64[q];
        }
    }
#pragma unroll
    for (int q = 0; q < 6; q++) cq[q] = (T)c64[q];
    diag = (T)d;
    mask = m;
}

#define NB_LINE_LOOP(v)                                                                                            \
    const int lane = threadIdx.x & 31, warpId = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;                      \
    const int nWarps = (gridDim.x * blockDim.x) >> 5;                                                              \
    for (int line = warpId; line < (v).nLines; line += nWarps)                                                     \
        for (int f = lane; f < (v).lineLen; f += 32)

static inline int Blocks(const LevelView &v) { return LineGrid(v.nLines > 0 ? v.nLines : 1, 148 * 8); }

// ---------------------------------------------------------------------------------------------------------------
// coarse cell types: an interior coarse cell is Dirichlet (EMPTY) if any child is, else FLUID if any child is,
// else SOLID (Neumann); a coarse ring cell on one face is Dirichlet if any of its ring children is Dirichlet or
// FLUID, else SOLID; ring edges and corners are SOLID.
// ---------------------------------------------------------------------------------------------------------------
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
        // child index ranges along each axis (fine ring index when the coarse index is on the ring)
        int ia[2], ja[2], ka[2], ni = 0, nj = 0, nk = 0;
        auto kids = [](int C, int Nc, int Nf, int *out, int &cnt) {
            if (C == 0) { out[0] = 0; cnt = 1; return; }
            if (C == Nc - 1) { out[0] = Nf - 1; cnt = 1; return; }
            out[0] = 2 * C - 1;
            cnt = 1;
            if (2 * C <= Nf - 2) out[cnt++] = 2 * C;
        };
        kids(I, cv.Ny, f.Ny, ia, ni);
        kids(J, cv.Nx, f.Nx, ja, nj);
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
// smoother
// ---------------------------------------------------------------------------------------------------------------
template <typename T, bool kFirst>
__global__ void __launch_bounds__(kBlock) k_smooth(LevelView v, const T *__restrict__ r, T *e, int colour)
{
    NB_LINE_LOOP(v)
    {
        int i, j, k;
        long long c;
        LineCell(v, line, f, i, j, k, c);
        if (v.types[c] != FLUID) continue;
        const int col = (i + j + k) & 1;
        if (kFirst)
        {
            if (col == 0)
            {
                T cq[6], diag;
                unsigned m;
                LevelStencil<T>(v, i, j, k, c, cq, diag, m);
                e[c] = diag != (T)0 ? r[c] / diag : (T)0;
            }
            else
                e[c] = (T)0;
            continue;
        }
        if (col != colour) continue;
        T cq[6], diag;
        unsigned m;
        LevelStencil<T>(v, i, j, k, c, cq, diag, m);
        T s = r[c];
        const int nq = v.dim == 3 ? 6 : 4;
#pragma unroll
        for (int q = 0; q < 6; q++)
            if (q < nq && (m >> q & 1u)) s += cq[q] * e[c + NbrOffset(v, q)];
        e[c] = diag != (T)0 ? s / diag : (T)0;
    }
}

template <typename T> void LaunchSmoothFirst(const LevelView &v, const T *r, T *e, cudaStream_t st)
{
    if (v.nLines <= 0) return;
    NB_COUNT_LAUNCH();
    k_smooth<T, true><<<Blocks(v), kBlock, 0, st>>>(v, r, e, 0);
}

template <typename T> void LaunchSmooth(const LevelView &v, const T *r, T *e, int colour, cudaStream_t st)
{
    if (v.nLines <= 0) return;
    NB_COUNT_LAUNCH();
    k_smooth<T, false><<<Blocks(v), kBlock, 0, st>>>(v, r, e, colour);
}

// res = r - M e
template <typename T>
__global__ void __launch_bounds__(kBlock) k_level_residual(LevelView v, const T *__restrict__ r,
                                                           const T *__restrict__ e, T *__restrict__ res)
{
    NB_LINE_LOOP(v)
    {
        int i, j, k;
        long long c;
        LineCell(v, line, f, i, j, k, c);
        if (v.types[c] != FLUID) continue;
        T cq[6], diag;
        unsigned m;
        LevelStencil<T>(v, i, j, k, c, cq, diag, m);
        T s = diag * e[c];
        const int nq = v.dim == 3 ? 6 : 4;
#pragma unroll
        for (int q = 0; q < 6; q++)
            if (q < nq && (m >> q & 1u)) s -= cq[q] * e[c + NbrOffset(v, q)];
        res[c] = r[c] - s;
    }
}

template <typename T> void LaunchLevelResidual(const LevelView &v, const T *r, const T *e, T *res, cudaStream_t st)
{
    if (v.nLines <= 0) return;
    NB_COUNT_LAUNCH();
    k_level_residual<T><<<Blocks(v), kBlock, 0, st>>>(v, r, e, res);
}

// ---------------------------------------------------------------------------------------------------------------
// transfers. The prolongation is trilinear except at Neumann boundaries: a coarse contributor that is SOLID hands
// its weight to the child's parent (a constant extrapolation across the wall, the reflection a zero-gradient
// boundary asks for), a Dirichlet contributor keeps its zero. The restriction is the exact transpose.
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
__global__ void __launch_bounds__(kBlock) k_restrict(LevelView fv, LevelView cv, const T *__restrict__ res,
                                                     T *__restrict__ rc)
{
    NB_LINE_LOOP(cv)
    {
        int I, J, K;
        long long c;
        LineCell(cv, line, f, I, J, K, c);
        if (cv.types[c] != FLUID) continue;
        T s = (T)0;
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
                    s += wij * t;
                }
                else
                    s += wij * res[rowBase];
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
                    const int si = ci ? 1 : -1, sj = cj ? 1 : -1, sk = ck ? 1 : -1;
                    const T extra = SolidWeight<T>(cv, I, J, K, si, sj, sk);
                    if (extra != (T)0) s += extra * res[(long long)a * fv.sI + (long long)b * fv.sJ + d];
                }
        rc[c] = s;
    }
}

template <typename T>
void LaunchRestrict(const LevelView &fine, const LevelView &coarse, const T *resFine, T *rCoarse, cudaStream_t st)
{
    if (coarse.nLines <= 0) return;
    NB_COUNT_LAUNCH();
    k_restrict<T><<<Blocks(coarse), kBlock, 0, st>>>(fine, coarse, resFine, rCoarse);
}

template <typename T>
__global__ void __launch_bounds__(kBlock) k_prolong(LevelView fv, LevelView cv, const T *__restrict__ ec, T *ef)
{
    NB_LINE_LOOP(fv)
    {
        int a, b, d;
        long long c;
        LineCell(fv, line, f, a, b, d, c);
        if (fv.types[c] != FLUID) continue;
        const int A = (a + 1) >> 1, B = (b + 1) >> 1;
        const int D = fv.dim == 3 ? (d + 1) >> 1 : 0;
        const int si = (a & 1) ? -1 : 1, sj = (b & 1) ? -1 : 1, sk = (d & 1) ? -1 : 1;
        const T wv[2] = {(T)0.75, (T)0.25};
        const long long parent = (long long)A * cv.sI + (long long)B * cv.sJ + D;
        T s = (T)0, extra = (T)0;
        const int nk = fv.dim == 3 ? 2 : 1;
        for (int di = 0; di < 2; di++)
            for (int dj = 0; dj < 2; dj++)
                for (int dk = 0; dk < nk; dk++)
                {
                    const long long cc = parent + (long long)(di * si) * cv.sI + (long long)(dj * sj) * cv.sJ + dk * sk;
                    const T w = wv[di] * wv[dj] * (fv.dim == 3 ? wv[dk] : (T)1);
                    if ((di | dj | dk) && cv.types[cc] == SOLID) extra += w; // Neumann: the parent's value
                    else s += w * ec[cc];
                }
        ef[c] += s + extra * ec[parent];
    }
}

template <typename T>
void LaunchProlong(const LevelView &fine, const LevelView &coarse, const T *eCoarse, T *eFine, cudaStream_t st)
{
    if (fine.nLines <= 0) return;
    NB_COUNT_LAUNCH();
    k_prolong<T><<<Blocks(fine), kBlock, 0, st>>>(fine, coarse, eCoarse, eFine);
}

// ---------------------------------------------------------------------------------------------------------------
// coarsest level: `sweeps` forward red-black pairs then as many backward black-red pairs, from zero, in one CTA
// ---------------------------------------------------------------------------------------------------------------
template <typename T>
__device__ void CoarseHalf(const LevelView &v, const T *r, T *e, int colour, int first)
{
    for (long long c = threadIdx.x; c < v.cells; c += blockDim.x)
    {
        const int k = (int)(c % v.Nz);
        const long long rr = c / v.Nz;
        const int j = (int)(rr % v.Nx), i = (int)(rr / v.Nx);
        if (i == 0 || i == v.Ny - 1 || j == 0 || j == v.Nx - 1) continue;
        if (v.dim == 3 && (k == 0 || k == v.Nz - 1)) continue;
        if (v.types[c] != FLUID) continue;
        const int col = (i + j + k) & 1;
        if (first && col != colour) { e[c] = (T)0; continue; }
        if (col != colour) continue;
        T cq[6], diag;
        unsigned m;
        LevelStencil<T>(v, i, j, k, c, cq, diag, m);
        T s = r[c];
        if (!first)
        {
            const int nq = v.dim == 3 ? 6 : 4;
            for (int q = 0; q < nq; q++)
                if (m >> q & 1u) s += cq[q] * e[c + NbrOffset(v, q)];
        }
        e[c] = diag != (T)0 ? s / diag : (T)0;
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
__global__ void __launch_bounds__(kBlock) k_dot(LevelView v, const T *__restrict__ r, const T *__restrict__ z,
                                                Reducer R, int base)
{
    double acc[3] = {0.0, 0.0, 0.0};
    NB_LINE_LOOP(v)
    {
        int i, j, k;
        long long c;
        LineCell(v, line, f, i, j, k, c);
        const double rv = (double)r[c], zv = (double)z[c];
        acc[0] += rv * zv;
        acc[1] += zv;
        acc[2] += rv;
    }
    GridReduce<3>(R, acc, base);
}

template <typename T>
void LaunchDot(const LevelView &v, const T *r, const T *z, const Reducer &R, int base, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_dot<T><<<LineGrid(v.nLines > 0 ? v.nLines : 1, R.maxBlocks), kBlock, 0, st>>>(v, r, z, R, base);
}

__device__ __forceinline__ double RzEff(const double *S, int base, int n, int singular)
{
    return singular ? S[base] - (S[base + 1] / (double)n) * S[base + 2] : S[base];
}

template <typename T, bool kExact>
__global__ void __launch_bounds__(kBlock) k_update_p_apply(LevelView v, const T *__restrict__ z,
                                                           const T *__restrict__ pIn, T *__restrict__ pOut,
                                                           T *__restrict__ q, Reducer R, const double *S, int first,
                                                           int baseNew, int baseOld, int n, int singular, int slotPQ)
{
    const double beta = first ? 0.0 : RzEff(S, baseNew, n, singular) / RzEff(S, baseOld, n, singular);
    const T b = (T)beta;
    const T mean = singular ? (T)(S[baseNew + 1] / (double)n) : (T)0;
    double acc[1] = {0.0};
    NB_LINE_LOOP(v)
    {
        int i, j, k;
        long long c;
        LineCell(v, line, f, i, j, k, c);
        if (v.types[c] != FLUID) continue;
        T cq[6], diag;
        unsigned m;
        Stencil<T, kExact>(v, i, j, k, c, cq, diag, m);
        const T pc = (z[c] - mean) + b * pIn[c];
        T s = diag * pc;
        const int nq = v.dim == 3 ? 6 : 4;
#pragma unroll
        for (int qq = 0; qq < 6; qq++)
        {
            if (qq >= nq || !(m >> qq & 1u)) continue;
            const long long nb = c + NbrOffset(v, qq);
            T pn;
            if (singular)
            {
                const int ni = i + (qq == 0) - (qq == 1), nj = j + (qq == 2) - (qq == 3), nk = k + (qq == 4) - (qq == 5);
                pn = OnRing(v, ni, nj, nk) ? (T)0 : (z[nb] - mean) + b * pIn[nb];
            }
            else
                pn = z[nb] + b * pIn[nb];
            s -= cq[qq] * pn;
        }
        pOut[c] = pc;
        q[c] = s;
        acc[0] += (double)pc * (double)s;
    }
    GridReduce<1>(R, acc, slotPQ);
}

template <typename T>
void LaunchUpdatePApply(const LevelView &v, const T *z, const T *pIn, T *pOut, T *q, const Reducer &R,
                        const double *S, int first, int baseNew, int baseOld, int n, int singular, int slotPQ,
                        int exact, cudaStream_t st)
{
    const int blocks = LineGrid(v.nLines > 0 ? v.nLines : 1, R.maxBlocks);
    if (exact)
        {
            NB_COUNT_LAUNCH();
            k_update_p_apply<T, true><<<blocks, kBlock, 0, st>>>(v, z, pIn, pOut, q, R, S, first, baseNew, baseOld, n,
                                                                 singular, slotPQ);
        }
    else
        {
            NB_COUNT_LAUNCH();
            k_update_p_apply<T, false><<<blocks, kBlock, 0, st>>>(v, z, pIn, pOut, q, R, S, first, baseNew, baseOld, n,
                                                                  singular, slotPQ);
        }
}

template <typename T>
__global__ void __launch_bounds__(kBlock) k_update_xr(LevelView v, T *__restrict__ x, T *__restrict__ r,
                                                      const T *__restrict__ p, const T *__restrict__ q, Reducer R,
                                                      const double *S, int baseRZ, int n, int singular, int slotPQ,
                                                      int slotRR)
{
    const double alpha = RzEff(S, baseRZ, n, singular) / S[slotPQ];
    const T a = (T)alpha;
    double acc[1] = {0.0};
    NB_LINE_LOOP(v)
    {
        int i, j, k;
        long long c;
        LineCell(v, line, f, i, j, k, c);
        const T pv = p[c];
        if (pv == (T)0 && q[c] == (T)0) { const double rv = (double)r[c]; acc[0] += rv * rv; continue; }
        x[c] += a * pv;
        const T rn = r[c] - a * q[c];
        r[c] = rn;
        acc[0] += (double)rn * (double)rn;
    }
    GridReduce<1>(R, acc, slotRR);
}

template <typename T>
void LaunchUpdateXR(const LevelView &v, T *x, T *r, const T *p, const T *q, const Reducer &R, const double *S,
                    int baseRZ, int n, int singular, int slotPQ, int slotRR, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_update_xr<T><<<LineGrid(v.nLines > 0 ? v.nLines : 1, R.maxBlocks), kBlock, 0, st>>>(
        v, x, r, p, q, R, S, baseRZ, n, singular, slotPQ, slotRR);
}

template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kBlock) k_scale_copy(LevelView v, const Tin *x, Tout *y, double s)
{
    NB_LINE_LOOP(v)
    {
        int i, j, k;
        long long c;
        LineCell(v, line, f, i, j, k, c);
        if (v.types[c] != FLUID) continue;
        y[c] = (Tout)((double)x[c] * s);
    }
}

template <typename Tin, typename Tout>
void LaunchScaleCopy(const LevelView &v, const Tin *x, Tout *y, double s, cudaStream_t st)
{
    if (v.nLines <= 0) return;
    NB_COUNT_LAUNCH();
    k_scale_copy<Tin, Tout><<<Blocks(v), kBlock, 0, st>>>(v, x, y, s);
}

// ---- instantiations ----
#define NB_INST(T)                                                                                                 \
    template void LaunchSmoothFirst<T>(const LevelView &, const T *, T *, cudaStream_t);                           \
    template void LaunchSmooth<T>(const LevelView &, const T *, T *, int, cudaStream_t);                           \
    template void LaunchLevelResidual<T>(const LevelView &, const T *, const T *, T *, cudaStream_t);              \
    template void LaunchRestrict<T>(const LevelView &, const LevelView &, const T *, T *, cudaStream_t);           \
    template void LaunchProlong<T>(const LevelView &, const LevelView &, const T *, T *, cudaStream_t);            \
    template void LaunchCoarseSolve<T>(const LevelView &, const T *, T *, int, cudaStream_t);                      \
    template void LaunchDot<T>(const LevelView &, const T *, const T *, const Reducer &, int, cudaStream_t);       \
    template void LaunchUpdatePApply<T>(const LevelView &, const T *, const T *, T *, T *, const Reducer &,        \
                                        const double *, int, int, int, int, int, int, int, cudaStream_t);          \
    template void LaunchUpdateXR<T>(const LevelView &, T *, T *, const T *, const T *, const Reducer &,            \
                                    const double *, int, int, int, int, int, cudaStream_t);
NB_INST(float)
NB_INST(double)
template void LaunchScaleCopy<double, float>(const LevelView &, const double *, float *, double, cudaStream_t);
template void LaunchScaleCopy<double, double>(const LevelView &, const double *, double *, double, cudaStream_t);
template void LaunchScaleCopy<float, double>(const LevelView &, const float *, double *, double, cudaStream_t);

} // namespace nb
