// IDP numbering without allocation: the same numbering as NumberUnknowns (nb_exact.cu; the reference's IDP loop,
// PressureSolver3D.cpp:133-139), with its per-line counts, offsets and scan state held in one fixed device array of
// this file instead of buffers the caller's context allocated.
//
// Who needs it: code that re-labels its cells every step (moving solids, a free surface) and renumbers the unknowns
// from device-resident cell types, but may not allocate at that point. Two cases are common: a host framework whose
// caching allocator already reserved the device memory (an outside cudaMalloc can fail, or fragment that pool), and a
// stepping loop running other streams beside this one, where cudaFree would stall the whole device because it
// synchronizes it. This entry point makes no cudaMalloc, cudaFree or allocating library call; its scratch memory
// exists once per device, for the lifetime of the process.
//
// Set-up: the first call on a device looks up that device's address of the scratch array (cudaGetSymbolAddress),
// with the device current, and notes the context it belongs to; a call that finds another context current (the
// device was reset since) looks the address up again. That lookup may load this library's device code onto the
// device, so make the first call on each device, and the first after a reset, before any stream capture begins.
//
// The scratch is shared by all callers on a device: two calls that overlap in time on one device (from different
// streams or host threads) race on it and corrupt each other's results. Calls that follow each other on one stream
// are ordered and safe.
#include "nb_solver.h"

#include <mutex>

namespace nb
{

namespace
{

// Up to 2^18 lines: 3D grids with (Ny-2)*(Nx-2) <= 262144 (e.g. a 512 x 512 interior cross-section, any Nz),
// 2D grids with Ny-2 <= 262144. Layout in ints: counts[kMaxLines] | offsets[kMaxLines + 1] | pad | ticket | pad.
constexpr int kOffsetsAt = kNoAllocMaxLines;
constexpr int kTicketAt = 2 * kNoAllocMaxLines + 64; // 256-byte aligned
constexpr int kScratchInts = kTicketAt + 64;

static __device__ __align__(256) int g_numberingScratch[kScratchInts];

constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
int *g_scratchAddr[kMaxDevices] = {};
void *g_scratchCtx[kMaxDevices] = {}; // the context the address belongs to

// The driver context current on this thread (cuCtxGetCurrent, reached through the runtime's entry-point query so
// that the library needs no link to the driver library), or null when it cannot be read.
void *CurrentContext()
{
    typedef int (*GetCurrent)(void **);
    static GetCurrent fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return (GetCurrent)f;
    }();
    void *c = nullptr;
    if (!fn || fn(&c) != 0) return nullptr;
    return c;
}

// The current device's address of the scratch array, looked up on the first call for the device, and again when
// the device's context is no longer the one it was looked up in (after a cudaDeviceReset the old address would
// point into a context that no longer exists).
int *ScratchAddress(int device)
{
    if (device < 0 || device >= kMaxDevices) throw InputError("device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setupMutex);
    void *ctx = CurrentContext();
    if (!g_scratchAddr[device] || !ctx || ctx != g_scratchCtx[device])
    {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_numberingScratch);
        if (e != cudaSuccess) throw CudaError("cudaGetSymbolAddress(numbering scratch)", e);
        g_scratchAddr[device] = (int *)p;
        g_scratchCtx[device] = CurrentContext();
    }
    return g_scratchAddr[device];
}

constexpr int kScanItems = 8; // counts per thread per tile of the scan

// Count the FLUID cells of each line (one warp per line, ballots over 32 cells at a time); the block that finishes
// last then turns the counts into exclusive offsets and writes the total to *nOut.
__global__ void __launch_bounds__(kBlock) k_count_scan_static(LevelView v, int *scratch, int32_t *nOut)
{
    int *counts = scratch;
    int *offsets = scratch + kOffsetsAt;
    unsigned *ticket = (unsigned *)(scratch + kTicketAt);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int line = gw; line < v.nLines; line += nw)
    {
        int cnt = 0;
        for (int f0 = 0; f0 < v.lineLen; f0 += 32)
        {
            const int f = f0 + lane;
            int i, j, k;
            long long c;
            LineCell(v, line, f < v.lineLen ? f : 0, i, j, k, c);
            cnt += __popc(__ballot_sync(0xffffffffu, f < v.lineLen && v.types[c] == FLUID));
        }
        if (lane == 0) counts[line] = cnt;
    }

    __shared__ bool s_last;
    __shared__ int s_warpSum[kWarps];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();

    // exclusive scan of counts[0, nLines) in tiles of kBlock * kScanItems, carrying the running total
    int carry = 0;
    for (int base = 0; base < v.nLines; base += kBlock * kScanItems)
    {
        const int first = base + threadIdx.x * kScanItems;
        int item[kScanItems], own = 0;
        for (int q = 0; q < kScanItems; q++)
        {
            item[q] = first + q < v.nLines ? __ldcg(counts + first + q) : 0;
            own += item[q];
        }
        int incl = own; // inclusive scan of `own` across the warp
        for (int d = 1; d < 32; d <<= 1)
        {
            const int t = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += t;
        }
        if (lane == 31) s_warpSum[warp] = incl;
        __syncthreads();
        int before = carry, tileTotal = 0;
        for (int w = 0; w < kWarps; w++)
        {
            if (w < warp) before += s_warpSum[w];
            tileTotal += s_warpSum[w];
        }
        before += incl - own;
        for (int q = 0; q < kScanItems; q++)
        {
            if (first + q < v.nLines) offsets[first + q] = before;
            before += item[q];
        }
        carry += tileTotal;
        __syncthreads(); // s_warpSum is rewritten by the next tile
    }
    if (threadIdx.x == 0)
    {
        offsets[v.nLines] = carry;
        *nOut = carry;
        *ticket = 0u;
    }
}

// idp[c] = offset of the line + rank of the cell among the line's FLUID cells; other cells keep -1.
__global__ void __launch_bounds__(kBlock) k_number_static(LevelView v, const int *scratch, int32_t *idp)
{
    const int *offsets = scratch + kOffsetsAt;
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int line = gw; line < v.nLines; line += nw)
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

} // namespace

void NumberUnknownsNoAlloc(int device, int dim, int Nx, int Ny, int Nz, const uint8_t *types, int32_t *idp,
                           int32_t *n, cudaStream_t st)
{
    if (dim != 2 && dim != 3) throw InputError("dim must be 2 or 3");
    if (dim == 2 && Nz != 1) throw InputError("a 2D grid has Nz = 1");
    if (Nx < 2 || Ny < 2 || Nz < 1 || (dim == 3 && Nz < 2)) throw InputError("grid too small");
    if (!types || !idp || !n) throw InputError("null device pointer");
    const long long cells = (long long)Nx * Ny * Nz;
    if (cells > 0x7fffffffLL) throw InputError("more than 2^31 - 1 cells: IDP numbers are 32-bit");
    LevelView v{};
    v.dim = dim;
    v.Nx = Nx;
    v.Ny = Ny;
    v.Nz = Nz;
    v.cells = cells;
    v.sI = dim == 3 ? (long long)Nx * Nz : Nx;
    v.sJ = dim == 3 ? Nz : 1;
    const long long lines = dim == 3 ? (long long)(Ny - 2) * (Nx - 2) : Ny - 2;
    v.lineLen = dim == 3 ? Nz - 2 : Nx - 2;
    v.lineDiv = dim == 3 && Nx > 2 ? Nx - 2 : 1;
    if (lines > kNoAllocMaxLines)
        throw InputError("grid has " + std::to_string(lines) + " interior lines; the allocation-free numbering "
                         "holds at most " + std::to_string(kNoAllocMaxLines) +
                         " (use nereus_b200_set_layout + nereus_b200_get_idp)");
    v.nLines = lines > 0 && v.lineLen > 0 ? (int)lines : 0;
    v.types = types;

    int *scratch = ScratchAddress(device);
    NB_CK(cudaMemsetAsync(idp, 0xFF, sizeof(int32_t) * (size_t)cells, st));
    if (v.nLines == 0)
    {
        NB_CK(cudaMemsetAsync(n, 0, sizeof(int32_t), st));
        return;
    }
    // the scan's completion ticket must start at zero (the last block also resets it, but a call that failed midway
    // would leave it set)
    NB_CK(cudaMemsetAsync(scratch + kTicketAt, 0, sizeof(unsigned), st));
    const int blocks = LineGrid(v.nLines, 148 * 8);
    NB_COUNT_LAUNCH();
    k_count_scan_static<<<blocks, kBlock, 0, st>>>(v, scratch, n);
    NB_COUNT_LAUNCH();
    k_number_static<<<blocks, kBlock, 0, st>>>(v, scratch, idp);
    NB_CK(cudaGetLastError());
}

} // namespace nb
