// FLIP's re-labelling from particle positions on the device: FLIP3D::UpdateFluidCells
// (src/Methods/FLIP/FLIP3D.cpp:784-833) and FLIP2D::UpdateFluidCells (src/Methods/FLIP/FLIP2D.cpp:648-691), with
// MAC::ResetFluidCells (src/MAC.cpp:556-589). The labels come out byte for byte as the reference's serial loops leave
// them, so the pressure step that follows (set_layout) numbers and assembles the same system.
//
// The reference's three steps and how they run here (five launches on one stream, no allocation, no host wait, so a
// caller may capture them in a graph):
//   1. reset: every cell that is not SOLID, INFLOW, OUTFLOW or PRESSURE becomes EMPTY. k_relabel_reset, 16 bytes per
//      thread; it also zeroes the pending-list counter and the skipped-particle count.
//   2. mark: each particle's cell, if EMPTY, becomes FLUID. k_relabel_mark, one wave of threads striding over the
//      particles four at a time, reading
//      x, y, z through a stride so that the reference's own Particle array (x, y, z at doubles 1..3 of 7) and plain
//      position arrays both serve. The index is the reference's (truncation of (x - origin) / dh toward zero, clamped
//      above); a particle more than one cell below the grid or with a non-finite coordinate, which the reference
//      would index outside its labels with, is skipped and counted.
//   3. hole filling: one pass over the interior in (i, j, k) order, IN PLACE: an EMPTY cell with >= 5 (3D) / >= 3
//      (2D) FLUID neighbours becomes FLUID, and a cell filled earlier in the pass counts for the later ones. So a cell
//      sees its upper neighbours (i+1, j+1, k+1) as they were before the pass and its lower ones (i-1, j-1, k-1) as
//      the pass left them. The result is the unique solution of that recurrence, which is what is computed here:
//        k_relabel_fill: one thread per interior cell, consecutive threads along the fast axis, whole columns per
//          block step. Filled cells get the
//          marker kFilled, which counts as FLUID for the cells above and not at all for the cells below (they read
//          the label from before the pass). A filled cell has at most one uncounted neighbour, so at most one of its
//          upper neighbours can continue a chain of fills: the thread walks up that chain at once. A cell still EMPTY
//          that could yet be filled once its lower neighbours are (the count with every EMPTY interior lower
//          neighbour taken as filled reaches the threshold) goes on a pending list.
//        k_relabel_settle: one block iterates over the pending list until a pass fills nothing. Every fill is
//          justified by neighbours that belong to the solution, and every cell of the solution not yet filled is on
//          the list, so the fixed point is the solution; each pass but the last fills at least one cell, which bounds
//          the passes by the list's length + 1. When the list outgrew the caller's scratch, the block runs the same
//          passes over every interior cell instead.
//        k_relabel_finish: kFilled -> FLUID.
#include "nb_solver.h"

#include <cstdint>

namespace nb
{

namespace
{

constexpr uint8_t kFilled = 0x80; // an EMPTY cell the hole pass filled, until k_relabel_finish
constexpr int kThreads = 256;
constexpr int kSettleThreads = 1024;
constexpr int kHeaderInts = 4; // scratch: [0] pending count, [1..3] unused, then the list

struct RelabelGrid
{
    int dim, Nx, Ny, Nz;       // Nz = 1 in 2D
    long long cells;
    long long sI, sJ;          // strides of i and j (2D: sJ = 1 is the march axis)
    int colsX;                 // interior columns along the second axis (3D: Nx - 2; 2D: 1)
    int nCols;                 // interior columns
    int march;                 // interior cells along the march axis (3D: Nz - 2; 2D: Nx - 2)
    int thr;                   // FLUID neighbours that fill a hole: 5 (3D), 3 (2D)
};

__device__ __forceinline__ uint8_t ResetByte(uint8_t b)
{
    return (b == SOLID || b == INFLOW || b == OUTFLOW || b == PRESSURE) ? b : (uint8_t)EMPTY;
}

__device__ __forceinline__ uint32_t ResetWord(uint32_t w)
{
    uint32_t o = 0;
#pragma unroll
    for (int s = 0; s < 32; s += 8) o |= (uint32_t)ResetByte((uint8_t)(w >> s)) << s;
    return o;
}

__device__ __forceinline__ uint32_t FinishWord(uint32_t w)
{
    uint32_t o = 0;
#pragma unroll
    for (int s = 0; s < 32; s += 8)
    {
        const uint8_t b = (uint8_t)(w >> s);
        o |= (uint32_t)(b == kFilled ? (uint8_t)FLUID : b) << s;
    }
    return o;
}

// A byte map over the whole label array: the bytes before the first 16-byte boundary and after the last one
// one at a time, the rest as uint4.
template <bool kFinish>
__device__ __forceinline__ void MapLabels(uint8_t *__restrict__ t, long long cells)
{
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nt = (long long)gridDim.x * blockDim.x;
    const long long mis = (long long)((16 - ((uintptr_t)t & 15)) & 15);
    const long long head = mis < cells ? mis : cells;
    const long long nvec = (cells - head) >> 4;
    for (long long c = tid; c < head; c += nt)
        t[c] = kFinish ? (t[c] == kFilled ? (uint8_t)FLUID : t[c]) : ResetByte(t[c]);
    uint4 *v = (uint4 *)(t + head);
    for (long long q = tid; q < nvec; q += nt)
    {
        uint4 x = v[q];
        if (kFinish)
        {
            x.x = FinishWord(x.x); x.y = FinishWord(x.y); x.z = FinishWord(x.z); x.w = FinishWord(x.w);
        }
        else
        {
            x.x = ResetWord(x.x); x.y = ResetWord(x.y); x.z = ResetWord(x.z); x.w = ResetWord(x.w);
        }
        v[q] = x;
    }
    for (long long c = head + (nvec << 4) + tid; c < cells; c += nt)
        t[c] = kFinish ? (t[c] == kFilled ? (uint8_t)FLUID : t[c]) : ResetByte(t[c]);
}

__global__ void __launch_bounds__(kThreads) k_relabel_reset(uint8_t *__restrict__ t, long long cells, int *hdr,
                                                            unsigned long long *skipped)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        hdr[0] = 0;
        if (skipped) *skipped = 0ull;
    }
    MapLabels<false>(t, cells);
}

__global__ void __launch_bounds__(kThreads) k_relabel_finish(uint8_t *__restrict__ t, long long cells)
{
    MapLabels<true>(t, cells);
}

// UpdateFluidCells' index of one coordinate (FLIP3D.cpp:796-802): trunc((x - origin) / dh), at most N - 1; -1 for a
// quotient at or below -1 or not finite (outside the labels in the reference). A quotient at or above N takes N - 1
// without a conversion.
// The quotient is first taken as (x - origin) * inv with inv = 1 / dh rounded, which is within 2^-51 |q| of the
// correctly rounded quotient q (two roundings of 2^-53 each, plus the one of q). Every decision below compares q with
// an integer (the truncation, -1, N), so where the product lies farther than that bound (2^-48 |q| here, with margin)
// from both integers around it, q lies strictly between the same two integers and every decision agrees; otherwise
// (and for a non-finite product) the exact IEEE division decides.
__device__ __forceinline__ int ParticleIndex(double x, double origin, double dh, double inv, int N)
{
    const double d = x - origin;
    double q = d * inv;
    const double fl = floor(q);
    const double tol = fabs(q) * 0x1p-48 + 0x1p-60;
    if (!(q - fl > tol && fl + 1.0 - q > tol)) q = d / dh;
    if (!(q > -1.0)) return -1;
    if (q >= (double)N) return N - 1;
    return (int)q;
}

constexpr int kMarkBatch = 4; // particles in flight per thread

__global__ void __launch_bounds__(kThreads, 4)
    k_relabel_mark(const double *__restrict__ px, const double *__restrict__ py, const double *__restrict__ pz,
                   long long count, long long stride, RelabelGrid g, double ox, double oy, double oz, double dh,
                   double inv, uint8_t *__restrict__ t, unsigned long long *skipped)
{
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nt = (long long)gridDim.x * blockDim.x;
    unsigned long long mine = 0;
    const long long step = nt * kMarkBatch;
    double x[kMarkBatch], y[kMarkBatch], z[kMarkBatch];
    // positions of particles p, p + nt, ..., p + 3 nt (the first one again past the end: it is in range)
    auto load = [&](long long p) {
#pragma unroll
        for (int b = 0; b < kMarkBatch; b++)
        {
            const long long o = (p + b * nt < count ? p + b * nt : p) * stride;
            x[b] = __ldg(px + o);
            y[b] = __ldg(py + o);
            z[b] = g.dim == 3 ? __ldg(pz + o) : 0.0;
        }
    };
    long long p0 = tid;
    if (p0 < count) load(p0);
    while (p0 < count)
    {
        long long c[kMarkBatch];
#pragma unroll
        for (int b = 0; b < kMarkBatch; b++)
        {
            const int i = ParticleIndex(y[b], oy, dh, inv, g.Ny);
            const int j = ParticleIndex(x[b], ox, dh, inv, g.Nx);
            const int k = g.dim == 3 ? ParticleIndex(z[b], oz, dh, inv, g.Nz) : 0;
            const bool live = p0 + b * nt < count;
            const bool out = (i | j | k) < 0;
            mine += live && out;
            c[b] = live && !out ? ((long long)i * g.Nx + j) * g.Nz + k : -1;
        }
        // the next batch's positions are in flight while this batch's labels are read and written
        const long long p1 = p0 + step;
        if (p1 < count) load(p1);
#pragma unroll
        for (int b = 0; b < kMarkBatch; b++)
            if (c[b] >= 0 && t[c[b]] == EMPTY) t[c[b]] = (uint8_t)FLUID;
        p0 = p1;
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, s);
    if (skipped && (threadIdx.x & 31) == 0 && mine) atomicAdd(skipped, mine);
}

// FLUID neighbours of interior cell c as the in-place pass sees them: the upper ones (c + sI, c + sJ, c + 1) only if
// FLUID before the pass, the lower ones if FLUID or filled by it. In 2D the sJ terms are the march axis's own, so
// they are left out (sJ = 1 = the +-1 terms).
__device__ __forceinline__ int FluidCount(const RelabelGrid &g, const uint8_t *t, long long c)
{
    int up = (t[c + g.sI] == FLUID) + (t[c + 1] == FLUID);
    const uint8_t a = t[c - g.sI], b = t[c - 1];
    int lo = (a == FLUID || a == kFilled) + (b == FLUID || b == kFilled);
    if (g.dim == 3)
    {
        up += t[c + g.sJ] == FLUID;
        const uint8_t d = t[c - g.sJ];
        lo += d == FLUID || d == kFilled;
    }
    return up + lo;
}

// The same count for the owner of cell c at (i, j, m), with `maybe`, its EMPTY interior lower neighbours (those that
// may still be filled), taken from ONE read of each lower neighbour. Other threads fill cells meanwhile; had the two
// figures come from separate reads, a neighbour filled between them would be in neither and c could be left out of
// both the fills and the pending list. From one read, every lower neighbour that belongs to the solution is either
// FLUID/filled (counted) or EMPTY (in `maybe`), so a cell of the solution that is not filled is always listed. The
// upper neighbours' "FLUID before the pass" never changes during the pass.
__device__ __forceinline__ int FluidCountOnce(const RelabelGrid &g, const uint8_t *t, long long c, int i, int j, int m,
                                              int &maybe)
{
    const volatile uint8_t *vt = t;
    int up = (t[c + g.sI] == FLUID) + (t[c + 1] == FLUID);
    const uint8_t a = vt[c - g.sI], b = vt[c - 1];
    int lo = (a == FLUID || a == kFilled) + (b == FLUID || b == kFilled);
    maybe = (i > 1 && a == EMPTY) + (m > 1 && b == EMPTY);
    if (g.dim == 3)
    {
        up += t[c + g.sJ] == FLUID;
        const uint8_t d = vt[c - g.sJ];
        lo += d == FLUID || d == kFilled;
        maybe += j > 1 && d == EMPTY;
    }
    return up + lo;
}

// Coordinates of cell c: (i, j, m) with m the march-axis index (k in 3D, j in 2D; j = 0 in 2D). Cells number
// below 2^31, so 32-bit arithmetic serves.
__device__ __forceinline__ void CellCoords(const RelabelGrid &g, long long c, int &i, int &j, int &m)
{
    const unsigned cu = (unsigned)c, sI = (unsigned)g.sI, sJ = (unsigned)g.sJ;
    i = (int)(cu / sI);
    const unsigned r = cu - (unsigned)i * sI;
    if (g.dim == 3)
    {
        j = (int)(r / sJ);
        m = (int)(r - (unsigned)j * sJ);
    }
    else
    {
        j = 0;
        m = (int)r;
    }
}

// Cell c was just filled. A filled cell has at most one neighbour that counts as non-FLUID, so at most one of its
// upper neighbours can still be EMPTY: if that one now reaches the threshold it is filled too, and the walk goes on
// from it. Every step fills a cell that was EMPTY, which bounds the walk by the number of interior cells.
__device__ __forceinline__ void ChaseUp(const RelabelGrid &g, uint8_t *t, long long c, int i, int j, int m)
{
    for (;;)
    {
        const int lastM = g.dim == 3 ? g.Nz - 2 : g.Nx - 2;
        long long u = -1;
        if (m < lastM && t[c + 1] == EMPTY) { u = c + 1; m++; }
        else if (g.dim == 3 && j < g.Nx - 2 && t[c + g.sJ] == EMPTY) { u = c + g.sJ; j++; }
        else if (i < g.Ny - 2 && t[c + g.sI] == EMPTY) { u = c + g.sI; i++; }
        if (u < 0 || FluidCount(g, t, u) < g.thr) return;
        t[u] = kFilled;
        c = u;
    }
}

// Interior cell number q (0 .. interior cells - 1) in (i, j, k) order.
__device__ __forceinline__ long long InteriorCell(const RelabelGrid &g, long long q)
{
    const unsigned qu = (unsigned)q, march = (unsigned)g.march;
    const unsigned col = qu / march;
    const int m = 1 + (int)(qu - col * march);
    const int i = 1 + (int)(col / (unsigned)g.colsX);
    const int j = g.dim == 3 ? 1 + (int)(col % (unsigned)g.colsX) : 0;
    return (g.dim == 3 ? ((long long)i * g.Nx + j) * g.Nz : (long long)i * g.Nx) + m;
}

// Each block step takes whole columns: `span` threads per column along the march axis (consecutive threads on
// consecutive cells), kThreads / span columns per step. A cell that reaches the threshold with the labels as this
// thread reads them is filled (and the chain above it followed); one that could still reach it once its EMPTY lower
// neighbours are filled goes on the pending list.
__global__ void __launch_bounds__(kThreads)
    k_relabel_fill(RelabelGrid g, uint8_t *t, int *hdr, int *list, int cap)
{
    const int span = g.march < kThreads ? g.march : kThreads;
    const int cpb = kThreads / span;
    const int lc = threadIdx.x / span, lm = threadIdx.x - lc * span;
    if (lc >= cpb) return;
    for (int col0 = blockIdx.x * cpb; col0 < g.nCols; col0 += gridDim.x * cpb)
    {
        const int col = col0 + lc;
        if (col >= g.nCols) return;
        const int i = 1 + col / g.colsX;
        const int j = g.dim == 3 ? 1 + (col - (i - 1) * g.colsX) : 0;
        const long long base = g.dim == 3 ? ((long long)i * g.Nx + j) * g.Nz : (long long)i * g.Nx;
        for (int m = 1 + lm; m <= g.march; m += span)
        {
            const long long c = base + m;
            if (t[c] != EMPTY) continue;
            int maybe = 0;
            const int f = FluidCountOnce(g, t, c, i, j, m, maybe);
            if (f >= g.thr)
            {
                t[c] = kFilled;
                ChaseUp(g, t, c, i, j, m);
                continue;
            }
            if (f + maybe >= g.thr)
            {
                const int slot = atomicAdd(hdr, 1);
                if (slot < cap) list[slot] = (int)c;
            }
        }
    }
}

__global__ void __launch_bounds__(kSettleThreads)
    k_relabel_settle(RelabelGrid g, uint8_t *t, const int *hdr, const int *list, int cap)
{
    __shared__ int changed;
    const int pending = hdr[0];
    const bool all = pending > cap; // the list overflowed: pass over every interior cell
    const long long n = all ? (long long)g.nCols * g.march : pending;
    for (long long pass = 0; pass <= n; pass++)
    {
        if (threadIdx.x == 0) changed = 0;
        __syncthreads();
        bool any = false;
        for (long long q = threadIdx.x; q < n; q += blockDim.x)
        {
            const long long c = all ? InteriorCell(g, q) : (long long)list[q];
            if (t[c] == EMPTY && FluidCount(g, t, c) >= g.thr)
            {
                t[c] = kFilled;
                int i, j, m;
                CellCoords(g, c, i, j, m);
                ChaseUp(g, t, c, i, j, m);
                any = true;
            }
        }
        if (any) changed = 1;
        __syncthreads();
        const bool more = changed != 0;
        __syncthreads();
        if (!more) break;
    }
}

int Blocks(long long work, int perBlock, int cap)
{
    long long b = (work + perBlock - 1) / perBlock;
    if (b < 1) b = 1;
    return (int)(b < cap ? b : cap);
}

} // namespace

size_t RelabelScratchBytes(int dim, int Nx, int Ny, int Nz)
{
    const long long nz = dim == 3 ? (long long)(Nz > 2 ? Nz - 2 : 0) : 1;
    const long long interior = (long long)(Nx > 2 ? Nx - 2 : 0) * (Ny > 2 ? Ny - 2 : 0) * nz;
    return (size_t)(kHeaderInts + interior) * sizeof(int);
}

void UpdateFluidCellsDevice(int dim, int Nx, int Ny, int Nz, double ox, double oy, double oz, double dh,
                            const double *px, const double *py, const double *pz, long long count, long long stride,
                            uint8_t *cellTypes, void *scratch, size_t scratchBytes, unsigned long long *skipped,
                            cudaStream_t st)
{
    if (dim != 2 && dim != 3) throw InputError("dim must be 2 or 3");
    const int nz = dim == 3 ? Nz : 1;
    if (Nx < 1 || Ny < 1 || nz < 1) throw InputError("bad sizes");
    const long long cells = (long long)Nx * Ny * nz;
    if (cells >= (1ll << 31)) throw InputError("at most 2^31 - 1 cells");
    if (!cellTypes || !scratch) throw InputError("null argument");
    if (count < 0) throw InputError("negative particle count");
    if (count > 0 && (!px || !py || (dim == 3 && !pz))) throw InputError("null particle coordinates");
    if (count > 0 && stride < 1) throw InputError("particle stride must be at least 1");
    if (!(dh > 0.0) || !std::isfinite(dh)) throw InputError("dh must be positive and finite");
    if (scratchBytes < kHeaderInts * sizeof(int) || ((uintptr_t)scratch & 3)) throw InputError("scratch too small or misaligned");

    RelabelGrid g;
    g.dim = dim; g.Nx = Nx; g.Ny = Ny; g.Nz = nz; g.cells = cells;
    g.sI = (long long)Nx * nz;
    g.sJ = dim == 3 ? nz : 1;
    g.colsX = dim == 3 ? (Nx > 2 ? Nx - 2 : 0) : 1;
    g.nCols = (Ny > 2 ? Ny - 2 : 0) * g.colsX;
    g.march = dim == 3 ? (nz > 2 ? nz - 2 : 0) : (Nx > 2 ? Nx - 2 : 0);
    g.thr = 2 * dim - 1;
    int *hdr = (int *)scratch;
    int *list = hdr + kHeaderInts;
    const long long capLL = (long long)(scratchBytes / sizeof(int)) - kHeaderInts;
    const int cap = (int)(capLL < (1ll << 31) - 1 ? capLL : (1ll << 31) - 1);

    int dev = 0, sms = 148;
    NB_CK(cudaGetDevice(&dev));
    NB_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    NB_COUNT_LAUNCH();
    k_relabel_reset<<<Blocks(cells / 16 + 1, kThreads, sms * 8), kThreads, 0, st>>>(cellTypes, cells, hdr, skipped);
    if (count > 0)
    {
        NB_COUNT_LAUNCH();
        k_relabel_mark<<<Blocks((count + kMarkBatch - 1) / kMarkBatch, kThreads, sms * 4), kThreads, 0, st>>>(
            px, py, pz, count, stride, g, ox, oy, oz, dh, 1.0 / dh, cellTypes, skipped);
    }
    if (g.nCols > 0 && g.march > 0)
    {
        NB_COUNT_LAUNCHES(3);
        const int span = g.march < kThreads ? g.march : kThreads;
        k_relabel_fill<<<Blocks(g.nCols, kThreads / span, sms * 8), kThreads, 0, st>>>(g, cellTypes, hdr, list, cap);
        k_relabel_settle<<<1, kSettleThreads, 0, st>>>(g, cellTypes, hdr, list, cap);
        k_relabel_finish<<<Blocks(cells / 16 + 1, kThreads, sms * 8), kThreads, 0, st>>>(cellTypes, cells);
    }
    NB_CK(cudaGetLastError());
}

} // namespace nb
