// Device-side building blocks shared by the B200 pressure-projection kernels: the level view (sizes, strides, cell
// types, spacing tables), the 5/7-point coefficients, line-parallel iteration and deterministic grid reductions.
//
// Grid layout (NEREUS MAC, src/headers/Core/MAC.h:235-254): cell (i,j,k) = (y,x,z) at (i*Nx + j)*Nz + k with the
// one-cell border ring included in Nx, Ny, Nz. The fast axis is k in 3D and j in 2D (Nz = 1). Work is split into
// "lines": one interior (i,j) pair in 3D, one interior row i in 2D; a warp walks one line 32 cells at a time, so
// every load of a field is a contiguous, coalesced run.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace nb
{

enum : int { FLUID = 0, SOLID = 1, EMPTY = 2, INFLOW = 3, PRESSURE = 4, OUTFLOW = 5 };

__host__ __device__ inline bool IsDirichlet(int t) { return t == EMPTY || t == PRESSURE; }

// One multigrid level (level 0 is the caller's grid).
struct LevelView
{
    int dim;            // 2 or 3
    int Nx, Ny, Nz;     // ring included; Nz = 1 in 2D
    long long cells;
    long long sI, sJ;   // strides of i and j (3D: Nx*Nz, Nz; 2D: Nx, 1)
    int nLines;         // interior lines: 3D (Ny-2)*(Nx-2), 2D (Ny-2)
    int lineLen;        // interior cells along the fast axis
    int lineDiv;        // 3D: Nx-2 (line -> i, j); 2D: unused
    const uint8_t *types;
    int stretched;      // coefficients from the tables; otherwise every face coefficient is `gamma`
    double gamma;
    const double *w[3]; // padded Width tables, entry n at [n+1] (n = -1..N)
    const double *g[3]; // padded FaceGap tables, entry n at [n+1] (n = -1..N-1)
    const float *w32[3];
    const float *ig32[3]; // 1 / FaceGap, FP32
};

// Cell of interior line `line`, fast offset f (0-based).
__device__ __forceinline__ void LineCell(const LevelView &v, int line, int f, int &i, int &j, int &k, long long &c)
{
    if (v.dim == 3)
    {
        i = 1 + line / v.lineDiv;
        j = 1 + line - (i - 1) * v.lineDiv;
        k = 1 + f;
    }
    else
    {
        i = 1 + line;
        j = 1 + f;
        k = 0;
    }
    c = (long long)i * v.sI + (long long)j * v.sJ + k;
}

__device__ __forceinline__ long long NbrOffset(const LevelView &v, int q)
{
    // (i+1, i-1, j+1, j-1, k+1, k-1), the reference's q order (PressureSolver3D.cpp:66-68)
    switch (q)
    {
    case 0: return v.sI;
    case 1: return -v.sI;
    case 2: return v.sJ;
    case 3: return -v.sJ;
    case 4: return 1;
    default: return -1;
    }
}

__device__ __forceinline__ bool OnRing(const LevelView &v, int i, int j, int k)
{
    return i == 0 || i == v.Ny - 1 || j == 0 || j == v.Nx - 1 || (v.dim == 3 && (k == 0 || k == v.Nz - 1));
}

__device__ __forceinline__ double Wd(const LevelView &v, int a, int n) { return v.w[a][n + 1]; }
__device__ __forceinline__ double Gp(const LevelView &v, int a, int n) { return v.g[a][n + 1]; }

// Face coefficients of cell (i,j,k) in the solver's precision. Level 0 in FP64 gets the reference's values
// bit for bit through CoefsExact (nb_exact.cu); the multigrid levels use this cheaper form.
template <typename T>
__device__ __forceinline__ void LevelCoefs(const LevelView &v, int i, int j, int k, T c[6])
{
    if (!v.stretched)
    {
#pragma unroll
        for (int q = 0; q < 6; q++) c[q] = (T)v.gamma;
        return;
    }
    if (v.dim == 2)
    {
        const T wx = (T)v.w32[0][j + 1], wy = (T)v.w32[1][i + 1];
        c[0] = wx * (T)v.ig32[1][i + 1];
        c[1] = wx * (T)v.ig32[1][i];
        c[2] = wy * (T)v.ig32[0][j + 1];
        c[3] = wy * (T)v.ig32[0][j];
        c[4] = c[5] = (T)0;
        return;
    }
    const T wx = (T)v.w32[0][j + 1], wy = (T)v.w32[1][i + 1], wz = (T)v.w32[2][k + 1];
    const T ax = wy * wz, ay = wx * wz, az = wx * wy;
    c[0] = ay * (T)v.ig32[1][i + 1];
    c[1] = ay * (T)v.ig32[1][i];
    c[2] = ax * (T)v.ig32[0][j + 1];
    c[3] = ax * (T)v.ig32[0][j];
    c[4] = az * (T)v.ig32[2][k + 1];
    c[5] = az * (T)v.ig32[2][k];
}

// Dirichlet ring factor FaceGap / (Width/2) (PressureSettings.h:307-310) at the level's resolution.
template <typename T>
__device__ __forceinline__ T LevelRingFactor(const LevelView &v, int i, int j, int k, int q)
{
    if (!v.stretched) return (T)2;
    const int a = q < 2 ? 1 : (q < 4 ? 0 : 2);
    const int n = q < 2 ? i : (q < 4 ? j : k);
    const int s = (q & 1) ? -1 : 1;
    const float gap = 1.0f / v.ig32[a][(s < 0 ? n - 1 : n) + 1];
    return (T)(gap / (0.5f * v.w32[a][n + 1]));
}

// The unit-form operator M = -A/scale at one FLUID cell: off-diagonals c_q toward FLUID neighbours (whose vector
// entries are zero off the unknowns), diagonal sum of fluid faces plus Dirichlet faces times their ring factor.
template <typename T>
__device__ __forceinline__ void LevelStencil(const LevelView &v, int i, int j, int k, long long c, T cq[6], T &diag,
                                             unsigned &fluidMask)
{
    LevelCoefs<T>(v, i, j, k, cq);
    const int nq = v.dim == 3 ? 6 : 4;
    T d = 0;
    unsigned m = 0;
#pragma unroll
    for (int q = 0; q < 6; q++)
    {
        if (q >= nq) break;
        const int t = v.types[c + NbrOffset(v, q)];
        if (t == FLUID)
        {
            d += cq[q];
            m |= 1u << q;
        }
        else if (IsDirichlet(t))
        {
            const int ni = i + (q == 0) - (q == 1), nj = j + (q == 2) - (q == 3), nk = k + (q == 4) - (q == 5);
            d += OnRing(v, ni, nj, nk) ? cq[q] * LevelRingFactor<T>(v, i, j, k, q) : cq[q];
        }
    }
    diag = d;
    fluidMask = m;
}

// ---- reductions ----
template <typename T>
__device__ __forceinline__ T WarpSum(T x)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

__device__ __forceinline__ double WarpMax(double x)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

// Deterministic grid-wide sums: each block writes its partial sums, the last block to finish adds the partials in
// block order and stores the totals in `out`. The result depends only on the launch shape, so a repeated solve is
// bit-identical (the reference checks repeat solves for exact equality, tests/suite_pressure.cpp:119-141).
struct Reducer
{
    double *partials;   // [slot][block], stride maxBlocks
    unsigned *counter;
    double *out;        // scalar slots
    int maxBlocks;
};

constexpr int kBlock = 256;            // threads per block of the line kernels
constexpr int kWarps = kBlock / 32;

// Block-reduce NV values held by every thread, then the last block finishes; out[slot0 + s] = total s.
// op 0 = sum, 1 = max.
template <int NV>
__device__ __forceinline__ void GridReduce(const Reducer &R, double (&val)[NV], int slot0, int op = 0)
{
    __shared__ double sh[NV][kWarps];
    __shared__ bool amLast;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < NV; s++)
    {
        double x = op == 0 ? WarpSum(val[s]) : WarpMax(val[s]);
        if (lane == 0) sh[s][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
#pragma unroll
        for (int s = 0; s < NV; s++)
        {
            double t = sh[s][0];
            for (int w = 1; w < kWarps; w++) t = op == 0 ? t + sh[s][w] : fmax(t, sh[s][w]);
            R.partials[(size_t)s * R.maxBlocks + blockIdx.x] = t;
        }
        __threadfence();
        const unsigned done = atomicAdd(R.counter, 1u);
        amLast = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (!amLast) return;
    __threadfence();
#pragma unroll
    for (int s = 0; s < NV; s++)
    {
        double t = op == 0 ? 0.0 : 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
        {
            const double pv = *((volatile double *)&R.partials[(size_t)s * R.maxBlocks + b]);
            t = op == 0 ? t + pv : fmax(t, pv);
        }
        t = op == 0 ? WarpSum(t) : WarpMax(t);
        if (lane == 0) sh[s][warp] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
#pragma unroll
        for (int s = 0; s < NV; s++)
        {
            double t = sh[s][0];
            for (int w = 1; w < kWarps; w++) t = op == 0 ? t + sh[s][w] : fmax(t, sh[s][w]);
            R.out[slot0 + s] = t;
        }
        *R.counter = 0u;
    }
}

// Grid size for a level's line kernels: enough blocks to cover the lines, at most a few waves of the 148 SMs.
inline int LineGrid(int nLines, int maxBlocks)
{
    int b = (nLines + kWarps - 1) / kWarps;
    if (b < 1) b = 1;
    return b < maxBlocks ? b : maxBlocks;
}

} // namespace nb
