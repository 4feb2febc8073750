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
    // Per-cell code of the level: bits 0-5 neighbour q is FLUID, bit 6 a neighbour is Dirichlet, bit 7 the cell is
    // an unknown (interior FLUID). Built once per layout (k_build_codes).
    const uint8_t *code;
    // Tiled iteration over the interior: a block of 32 x 8 threads covers 32 cells along the fast axis and 8 along
    // the mid axis and marches `slowChunk` steps along the slow axis. 3D: (fast, mid, slow) = (k, j, i);
    // 2D: (j, i, -) with slowLen = 1.
    int fastLen, midLen, slowLen, slowChunk;
    // Colour-split layout of the level's FP32 vectors (sRS = 0: the grid layout). Cell (i, j, k) of colour
    // c = (i+j+k) & 1 sits at c*sHalf + i*sPS + j*sRS + (k >> 1): each colour is an Ny x Nx x sRS array whose rows
    // hold the Nz/2 cells of that colour, padded with zeros to a multiple of 4.
    int sRS, sPS;
    long long sHalf;
    // Colour-split level: act[i * actTiles + t] != 0 when tile t of plane i (elements 1024 t .. 1024 t + 1023 of
    // either colour's plane, the cells one block of a quad kernel owns on that plane) holds an unknown; null: every
    // tile counts as holding one. A block whose planes' tiles hold none skips its work: its cells stay zero.
    const uint8_t *act;
    int actTiles;
    // The x (mid-axis) groups of the transfer from this level to the next coarser one, where that coarsening keeps
    // some x cells whole (a stretched 3D level); null: cells 2J-1 and 2J under coarse J, as along the other axes.
    // xp[j] per fine j: parent J (bits 0-14), the other x contributor (bits 15-29; J itself when the parent has one
    // child) and bit 30 when the parent has one child (x weights 1 and 0, else 3/4 and 1/4).
    // xr[J] per coarse J: first child (bits 0-14), bit 15 when J has two children, bit 16 when the group before J
    // has two (its second child gives J a quarter), bit 17 when the group after J has two (its first child does).
    const int *xp, *xr;
};

__device__ __forceinline__ int XpParent(int x) { return x & 0x7FFF; }
__device__ __forceinline__ int XpOther(int x) { return (x >> 15) & 0x7FFF; }
__device__ __forceinline__ bool XpSingle(int x) { return (x >> 30) & 1; }

// The fine x cells that coarse J gathers from, with their weights (zero weight: an unused slot at a valid index);
// slots 1 and 2 are J's children (slot 2 only when it has two)
template <typename T> __device__ __forceinline__ void XrTaps(int x, int (&b)[4], T (&w)[4], bool &two)
{
    const int f0 = x & 0x7FFF;
    two = (x >> 15) & 1;
    b[0] = (x >> 16) & 1 ? f0 - 1 : f0;
    w[0] = (x >> 16) & 1 ? (T)0.25 : (T)0;
    b[1] = f0;
    w[1] = two ? (T)0.75 : (T)1;
    b[2] = two ? f0 + 1 : f0;
    w[2] = two ? (T)0.75 : (T)0;
    b[3] = (x >> 17) & 1 ? f0 + (two ? 2 : 1) : f0;
    w[3] = (x >> 17) & 1 ? (T)0.25 : (T)0;
}

// Index of cell (i, j, k) in a level vector of the level's layout.
__device__ __forceinline__ long long VecIdx(const LevelView &v, int i, int j, int k)
{
    if (v.sRS)
        return (long long)((i + j + k) & 1) * v.sHalf + (long long)i * v.sPS + (long long)j * v.sRS + (k >> 1);
    return (long long)i * v.sI + (long long)j * v.sJ + k;
}

enum : unsigned { CODE_FLUID_MASK = 0x3Fu, CODE_DIRICHLET = 0x40u, CODE_UNKNOWN = 0x80u };

constexpr int kTileF = 32, kTileM = 8;

// Coordinates of this thread's cell at slow step s (0-based); false outside the interior.
__device__ __forceinline__ bool TileCell(const LevelView &v, int fo, int mo, int s, int &i, int &j, int &k,
                                         long long &c)
{
    if (fo >= v.fastLen || mo >= v.midLen) return false;
    if (v.dim == 3) { i = 1 + s; j = 1 + mo; k = 1 + fo; }
    else { i = 1 + mo; j = 1 + fo; k = 0; }
    c = (long long)i * v.sI + (long long)j * v.sJ + k;
    return true;
}

// Cell of colour `colour` ((i+j+k)&1) number `ho` along the fast axis of its line; false past the line's end.
__device__ __forceinline__ bool TileCellColour(const LevelView &v, int ho, int mo, int s, int colour, int &i, int &j,
                                               int &k, long long &c)
{
    if (mo >= v.midLen) return false;
    int f;
    if (v.dim == 3)
    {
        i = 1 + s;
        j = 1 + mo;
        f = (((colour ^ (i + j)) & 1) ? 1 : 2) + 2 * ho; // k with (i + j + k) & 1 == colour
        if (f > v.fastLen) return false;
        k = f;
    }
    else
    {
        i = 1 + mo;
        f = (((colour ^ i) & 1) ? 1 : 2) + 2 * ho;
        if (f > v.fastLen) return false;
        j = f;
        k = 0;
    }
    c = (long long)i * v.sI + (long long)j * v.sJ + k;
    return true;
}

inline dim3 TileGrid(const LevelView &v, bool half = false)
{
    const int f = half ? (v.fastLen + 1) / 2 : v.fastLen;
    dim3 g((unsigned)((f + kTileF - 1) / kTileF), (unsigned)((v.midLen + kTileM - 1) / kTileM),
           (unsigned)((v.slowLen + v.slowChunk - 1) / v.slowChunk));
    if (g.x == 0) g.x = 1;
    if (g.y == 0) g.y = 1;
    if (g.z == 0) g.z = 1;
    return g;
}

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

// The same stencil from the cell's code: no neighbour type is read unless a neighbour is Dirichlet.
template <typename T>
__device__ __forceinline__ void CodeStencil(const LevelView &v, int i, int j, int k, long long c, unsigned code,
                                            T cq[6], T &diag)
{
    LevelCoefs<T>(v, i, j, k, cq);
    const unsigned m = code & CODE_FLUID_MASK;
    T d = 0;
#pragma unroll
    for (int q = 0; q < 6; q++)
        if (m >> q & 1u) d += cq[q];
    if (code & CODE_DIRICHLET)
    {
        const int nq = v.dim == 3 ? 6 : 4;
        for (int q = 0; q < nq; q++)
        {
            const int t = v.types[c + NbrOffset(v, q)];
            if (IsDirichlet(t))
            {
                const int ni = i + (q == 0) - (q == 1), nj = j + (q == 2) - (q == 3), nk = k + (q == 4) - (q == 5);
                d += OnRing(v, ni, nj, nk) ? cq[q] * LevelRingFactor<T>(v, i, j, k, q) : cq[q];
            }
        }
    }
    diag = d;
}

// ---- cell pairs (3D levels with Nz even): cells (i, j, 2m) and (i, j, 2m+1) form an aligned pair; a plane is
//      Nx*Nz/2 consecutive pairs; thread t of a launch takes pair t of the plane and marches along i ----
constexpr int kPairThreads = 256;
constexpr int kPairS = 8;                  // planes a thread marches at most
constexpr long long kPairBlocks = 148 * 8; // blocks a launch aims for

// Planes per thread for `planes` planes of `perPlane` blocks each: about kPairBlocks blocks, 1 .. kPairS planes.
inline int MarchPlanes(long long planes, long long perPlane)
{
    const long long s = (planes * perPlane + kPairBlocks - 1) / kPairBlocks;
    return (int)(s < 1 ? 1 : (s > kPairS ? kPairS : s));
}

// The launch grid of a pair kernel; minS: at least this many planes per thread (the launches that end in a
// grid-wide sum keep their partial sums few).
inline dim3 PairGrid(const LevelView &v, int minS = 1)
{
    const long long P = v.sI / 2, perPlane = (P + kPairThreads - 1) / kPairThreads, planes = v.Ny - 2;
    int S = MarchPlanes(planes, perPlane);
    const int cap = (int)(planes > 1 ? planes : 1);
    const int m = minS < cap ? minS : cap;
    if (m > S) S = m;
    return dim3((unsigned)perPlane, (unsigned)((planes + S - 1) / S));
}

// Per-thread position of a pair kernel.
struct PairPos
{
    int lane;
    bool valid;     // false for the clamped threads past the plane's last pair (they still load and shuffle)
    int i0, i1;     // planes [i0, i1)
    int sI, sJ;
    int j, k0;      // row and first cell of the pair (k0 even)
    long long base; // cell index of the pair's first cell on plane i0
};

__device__ __forceinline__ PairPos PairStart(const LevelView &v, int bx, int by, int gy)
{
    PairPos p;
    const int P = (int)(v.sI >> 1);
    p.lane = threadIdx.x & 31;
    int q = bx * kPairThreads + threadIdx.x;
    p.valid = q < P;
    if (!p.valid) q = P - 1;
    // the launch's grid.y splits the Ny-2 interior planes into chunks of S (the host sized it); a block past the
    // last plane starts at the ring plane and marches none
    const int S = (v.Ny - 2 + gy - 1) / gy;
    p.i0 = min(1 + by * S, v.Ny - 1);
    p.i1 = min(p.i0 + S, v.Ny - 1);
    p.sI = (int)v.sI;
    p.sJ = (int)v.sJ;
    const int cin = 2 * q;
    p.j = cin / v.Nz;
    p.k0 = cin - p.j * v.Nz;
    p.base = (long long)p.i0 * v.sI + cin;
    return p;
}
__device__ __forceinline__ PairPos PairStart(const LevelView &v)
{
    return PairStart(v, (int)blockIdx.x, (int)blockIdx.y, (int)gridDim.y);
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
// bump: when not null, the last block adds 1 to *bump after storing the totals (the PCG iteration counter, which
// every block of the launch has read before any block can be the last).
// addSlot0 >= 0 (sums only): each total also adds out[addSlot0 + s], the totals an earlier launch left there.
// GridReduceB: the same over the blocks bid = 0 .. nblk-1 of one reduction (a batched launch runs one reduction per
// request, each over its own blocks and Reducer).
template <int NV>
__device__ __forceinline__ void GridReduceB(const Reducer &R, double (&val)[NV], int slot0, unsigned bid,
                                            unsigned nblk, int op = 0, int *bump = nullptr, int addSlot0 = -1)
{
    __shared__ double sh[NV][32];
    __shared__ bool amLast;
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = tid & 31, warp = tid >> 5, nwarp = (nthr + 31) >> 5;
#pragma unroll
    for (int s = 0; s < NV; s++)
    {
        double x = op == 0 ? WarpSum(val[s]) : WarpMax(val[s]);
        if (lane == 0) sh[s][warp] = x;
    }
    __syncthreads();
    if (tid == 0)
    {
#pragma unroll
        for (int s = 0; s < NV; s++)
        {
            double t = sh[s][0];
            for (int w = 1; w < nwarp; w++) t = op == 0 ? t + sh[s][w] : fmax(t, sh[s][w]);
            R.partials[(size_t)s * R.maxBlocks + bid] = t;
        }
        __threadfence();
        const unsigned done = atomicAdd(R.counter, 1u);
        amLast = (done == nblk - 1);
    }
    __syncthreads();
    if (!amLast) return;
    __threadfence();
#pragma unroll
    for (int s = 0; s < NV; s++)
    {
        // L2 loads (the partials were written and fenced by the other blocks; nothing of them sits in this SM's
        // L1), unrolled so that many are in flight at once
        double t = 0.0;
        const double *part = R.partials + (size_t)s * R.maxBlocks;
#pragma unroll 8
        for (unsigned b = tid; b < nblk; b += nthr)
        {
            const double pv = __ldcg(part + b);
            t = op == 0 ? t + pv : fmax(t, pv);
        }
        t = op == 0 ? WarpSum(t) : WarpMax(t);
        if (lane == 0) sh[s][warp] = t;
    }
    __syncthreads();
    if (tid == 0)
    {
#pragma unroll
        for (int s = 0; s < NV; s++)
        {
            double t = sh[s][0];
            for (int w = 1; w < nwarp; w++) t = op == 0 ? t + sh[s][w] : fmax(t, sh[s][w]);
            if (addSlot0 >= 0) t += __ldcg(R.out + addSlot0 + s);
            R.out[slot0 + s] = t;
        }
        if (bump) *bump += 1;
        *R.counter = 0u;
    }
}

template <int NV>
__device__ __forceinline__ void GridReduce(const Reducer &R, double (&val)[NV], int slot0, int op = 0,
                                           int *bump = nullptr, int addSlot0 = -1)
{
    GridReduceB<NV>(R, val, slot0, blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z),
                    gridDim.x * gridDim.y * gridDim.z, op, bump, addSlot0);
}

// The block coordinates of a launch's blocks within one request's grid: a single launch passes blockIdx and gridDim,
// a batched launch (blockIdx.z = the request's place in the active list) the same x and y.
struct Blk
{
    int x, y, gx, gy;
};
__device__ __forceinline__ Blk ThisBlk() { return Blk{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x, (int)gridDim.y}; }
__device__ __forceinline__ unsigned BlkId(const Blk &b) { return (unsigned)(b.x + b.gx * b.y); }
__device__ __forceinline__ unsigned BlkCount(const Blk &b) { return (unsigned)(b.gx * b.gy); }

// ---- programmatic dependent launch: a kernel launched by LaunchPdl may be scheduled while the previous kernel on
// its stream drains. It calls PdlWait() before reading anything an earlier kernel wrote (the wait returns once that
// grid has completed and its writes are visible), then PdlTrigger(), which lets the next kernel start launching in
// turn. A kernel launched plainly runs both as no-ops. ----
__device__ __forceinline__ void PdlWait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void PdlTrigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t LaunchPdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                             Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Grid size for a level's line kernels: enough blocks to cover the lines, at most a few waves of the 148 SMs.
inline int LineGrid(int nLines, int maxBlocks)
{
    int b = (nLines + kWarps - 1) / kWarps;
    if (b < 1) b = 1;
    return b < maxBlocks ? b : maxBlocks;
}

} // namespace nb
