// The coarse end of the multigrid V-cycle in one thread block: every level from `tailStart` down (at most a few
// thousand cells each) lives in shared memory, and the block runs their pre-smoothing, residual, restriction,
// coarsest sweeps, prolongation and post-smoothing back to back. It reads the restricted residual of the first tail
// level from global memory and writes that level's correction back; the finer levels' kernels on either side are
// unchanged. The operations are the ones of nb_kernels.cu (same stencil, transfers and colour order), so the
// V-cycle stays the same symmetric operator.
//
// What costs time here is latency, not bytes: each phase (one colour of a sweep, a residual, a transfer) is a short
// loop over a level's unknowns followed by a barrier. So
// - the per-colour lists of unknowns are built once per layout (k_tail_lists) and only copied in;
// - a uniform level sums its six neighbours unmasked (every vector is zero off the unknowns) and divides through a
//   per-level reciprocal table of the diagonal's half-units, computed once per launch;
// - the levels with at most 32 unknowns of each colour (the last two or three) run in warp 0 alone, with __syncwarp
//   between their phases instead of a block-wide barrier.
#include "nb_kernels.h"

#include <cstring>
#include <mutex>
#include <set>

namespace nb
{

constexpr int kTailThreads = 256;

template <typename T> struct TailLevel
{
    LevelView v;
    unsigned off;     // byte offset of the level's arrays in shared memory
    unsigned listOff; // entry offset of the level's list in the global list array
};

template <typename T> struct TailArgs
{
    TailLevel<T> lv[kMaxTailLevels];
    int nlev;
    const T *rIn; // residual of the first tail level (global)
    T *eOut;      // its correction (global)
    int pre, post, coarseSweeps;
    const unsigned *lists; // per level: its cells' entries, red unknowns from the front, black ones from the back
    const int *counts;     // [level][colour] unknowns
};

// The level's arrays in shared memory: r, e, res (T), then code, types and diagonal units (bytes), then the list of
// its unknowns (4 bytes each: red ones from the front, black ones from the back), each padded to 16 bytes.
template <typename T> __host__ __device__ inline unsigned LevelBytes(long long cells)
{
    const unsigned a = (unsigned)((cells * sizeof(T) + 15) / 16 * 16);
    const unsigned b = (unsigned)((cells + 15) / 16 * 16);
    const unsigned l = (unsigned)((cells * 4 + 15) / 16 * 16);
    return 3 * a + 3 * b + l;
}

template <typename T> struct SmemLevel
{
    LevelView v; // types/code point into shared memory
    T *r, *e, *res;
    uint8_t *du;    // uniform level: 0x80 | diagonal half-units at an unknown, 0 elsewhere
    unsigned *list; // packed (i << 20 | j << 10 | k) of the unknowns; red [0, nRed), black [cells - nBlack, cells)
    int nRed, nBlack;
    const double *inv; // 1 / (gamma/2 * units), entry 0 = 0
};

__device__ __forceinline__ void Unpack(unsigned x, int &i, int &j, int &k)
{
    i = (int)(x >> 20);
    j = (int)((x >> 10) & 1023u);
    k = (int)(x & 1023u);
}

template <typename T> __device__ __forceinline__ SmemLevel<T> Bind(const TailLevel<T> &tl, unsigned char *smem)
{
    SmemLevel<T> s;
    s.v = tl.v;
    const long long cells = tl.v.cells;
    const unsigned a = (unsigned)((cells * sizeof(T) + 15) / 16 * 16);
    const unsigned b = (unsigned)((cells + 15) / 16 * 16);
    unsigned char *base = smem + tl.off;
    s.r = (T *)base;
    s.e = (T *)(base + a);
    s.res = (T *)(base + 2 * a);
    s.v.code = base + 3 * a;
    s.v.types = base + 3 * a + b;
    s.du = base + 3 * a + 2 * b;
    s.list = (unsigned *)(base + 3 * a + 3 * b);
    s.nRed = s.nBlack = 0;
    s.inv = nullptr;
    return s;
}

// the t-th unknown of the given colour (0 red, 1 black, 2 both: red then black)
template <typename T> __device__ __forceinline__ unsigned ListAt(const SmemLevel<T> &L, int colour, int t)
{
    const long long cells = L.v.cells;
    if (colour == 0) return L.list[t];
    if (colour == 1) return L.list[cells - 1 - t];
    return t < L.nRed ? L.list[t] : L.list[cells - 1 - (t - L.nRed)];
}

template <typename T> __device__ __forceinline__ int ListLen(const SmemLevel<T> &L, int colour)
{
    return colour == 0 ? L.nRed : (colour == 1 ? L.nBlack : L.nRed + L.nBlack);
}

__device__ __forceinline__ void Decode(const LevelView &v, long long c, int &i, int &j, int &k)
{
    k = (int)(c % v.Nz);
    const long long r = c / v.Nz;
    j = (int)(r % v.Nx);
    i = (int)(r / v.Nx);
}

// A phase runs over the whole block (kWarp false) or over warp 0 alone (kWarp true), and ends with the matching
// barrier.
template <bool kWarp> __device__ __forceinline__ int PhaseStart() { return kWarp ? (int)(threadIdx.x & 31) : (int)threadIdx.x; }
template <bool kWarp> __device__ __forceinline__ int PhaseStride() { return kWarp ? 32 : (int)blockDim.x; }
template <bool kWarp> __device__ __forceinline__ void PhaseSync()
{
    if (kWarp) __syncwarp();
    else __syncthreads();
}

// the plain sum of a cell's neighbours on a uniform level (vectors are zero off the unknowns)
template <typename T> __device__ __forceinline__ T NbrSum(const LevelView &v, const T *e, long long c)
{
    const T s = (e[c + v.sI] + e[c - v.sI]) + (e[c + v.sJ] + e[c - v.sJ]);
    return v.dim == 3 ? s + (e[c + 1] + e[c - 1]) : s;
}

template <typename T, bool kWarp> __device__ void TSmooth(const SmemLevel<T> &L, int colour, bool first)
{
    const LevelView &v = L.v;
    const int n = ListLen(L, colour);
    const T g = (T)v.gamma;
    for (int t = PhaseStart<kWarp>(); t < n; t += PhaseStride<kWarp>())
    {
        int i, j, k;
        Unpack(ListAt(L, colour, t), i, j, k);
        const long long c = (long long)i * v.sI + (long long)j * v.sJ + k;
        if (!v.stretched)
        {
            T rhs = L.r[c];
            if (!first) rhs += g * NbrSum(v, L.e, c);
            L.e[c] = rhs * (T)L.inv[L.du[c] & 0x7Fu];
            continue;
        }
        const unsigned code = v.code[c];
        T cq[6], diag;
        CodeStencil<T>(v, i, j, k, c, code, cq, diag);
        T rhs = L.r[c];
        if (!first)
        {
            if (code & 1u) rhs += cq[0] * L.e[c + v.sI];
            if (code & 2u) rhs += cq[1] * L.e[c - v.sI];
            if (code & 4u) rhs += cq[2] * L.e[c + v.sJ];
            if (code & 8u) rhs += cq[3] * L.e[c - v.sJ];
            if (code & 16u) rhs += cq[4] * L.e[c + 1];
            if (code & 32u) rhs += cq[5] * L.e[c - 1];
        }
        L.e[c] = diag != (T)0 ? rhs / diag : (T)0;
    }
    PhaseSync<kWarp>();
}

template <typename T, bool kWarp> __device__ void TResidual(const SmemLevel<T> &L)
{
    const LevelView &v = L.v;
    const int n = ListLen(L, 2);
    const T g = (T)v.gamma, hg = (T)0.5 * (T)v.gamma;
    for (int t = PhaseStart<kWarp>(); t < n; t += PhaseStride<kWarp>())
    {
        int i, j, k;
        Unpack(ListAt(L, 2, t), i, j, k);
        const long long c = (long long)i * v.sI + (long long)j * v.sJ + k;
        if (!v.stretched)
        {
            L.res[c] = L.r[c] - (hg * (T)(L.du[c] & 0x7Fu) * L.e[c] - g * NbrSum(v, L.e, c));
            continue;
        }
        const unsigned code = v.code[c];
        T cq[6], diag;
        CodeStencil<T>(v, i, j, k, c, code, cq, diag);
        T s = diag * L.e[c];
        if (code & 1u) s -= cq[0] * L.e[c + v.sI];
        if (code & 2u) s -= cq[1] * L.e[c - v.sI];
        if (code & 4u) s -= cq[2] * L.e[c + v.sJ];
        if (code & 8u) s -= cq[3] * L.e[c - v.sJ];
        if (code & 16u) s -= cq[4] * L.e[c + 1];
        if (code & 32u) s -= cq[5] * L.e[c - 1];
        L.res[c] = L.r[c] - s;
    }
    PhaseSync<kWarp>();
}

template <typename T>
__device__ __forceinline__ T TSolidWeight(const LevelView &cv, int I, int J, int K, int si, int sj, int sk)
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

template <typename T, bool kWarp> __device__ void TRestrict(const SmemLevel<T> &F, const SmemLevel<T> &C)
{
    const LevelView &fv = F.v, &cv = C.v;
    const int n = ListLen(C, 2);
    for (int t = PhaseStart<kWarp>(); t < n; t += PhaseStride<kWarp>())
    {
        int I, J, K;
        Unpack(ListAt(C, 2, t), I, J, K);
        const long long c = (long long)I * cv.sI + (long long)J * cv.sJ + K;
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
                    for (int dk = 0; dk < 4; dk++)
                    {
                        const int d = 2 * K - 2 + dk;
                        if (d <= fv.Nz - 1) t += wt[dk] * F.res[rowBase + d];
                    }
                    acc += wij * t;
                }
                else
                    acc += wij * F.res[rowBase];
            }
        }
        const int nz = fv.dim == 3 ? 2 : 1;
        for (int ci = 0; ci < 2; ci++)
            for (int cj = 0; cj < 2; cj++)
                for (int ck = 0; ck < nz; ck++)
                {
                    const int a = 2 * I - 1 + ci, b = 2 * J - 1 + cj, d = fv.dim == 3 ? 2 * K - 1 + ck : 0;
                    if (a > fv.Ny - 2 || b > fv.Nx - 2 || (fv.dim == 3 && d > fv.Nz - 2)) continue;
                    const T extra = TSolidWeight<T>(cv, I, J, K, ci ? 1 : -1, cj ? 1 : -1, ck ? 1 : -1);
                    if (extra != (T)0) acc += extra * F.res[(long long)a * fv.sI + (long long)b * fv.sJ + d];
                }
        C.r[c] = acc;
    }
    PhaseSync<kWarp>();
}

template <typename T, bool kWarp> __device__ void TProlong(const SmemLevel<T> &F, const SmemLevel<T> &C)
{
    const LevelView &fv = F.v, &cv = C.v;
    const int n = ListLen(F, 2);
    for (int t = PhaseStart<kWarp>(); t < n; t += PhaseStride<kWarp>())
    {
        int a, b, d;
        Unpack(ListAt(F, 2, t), a, b, d);
        const long long c = (long long)a * fv.sI + (long long)b * fv.sJ + d;
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
                    if ((di | dj | dk) && cv.types[cc] == SOLID) extra += w;
                    else acc += w * C.e[cc];
                }
        F.e[c] += acc + extra * C.e[parent];
    }
    PhaseSync<kWarp>();
}

// The descent through level l: the first sweep from zero, further sweeps, the residual and its restriction.
template <typename T, bool kWarp>
__device__ void TDown(const SmemLevel<T> &F, const SmemLevel<T> &C, int pre)
{
    TSmooth<T, kWarp>(F, 0, true);
    TSmooth<T, kWarp>(F, 1, false);
    for (int s = 1; s < pre; s++)
    {
        TSmooth<T, kWarp>(F, 0, false);
        TSmooth<T, kWarp>(F, 1, false);
    }
    TResidual<T, kWarp>(F);
    TRestrict<T, kWarp>(F, C);
}

// The coarsest level: symmetric sweep pairs from zero.
template <typename T, bool kWarp> __device__ void TCoarsest(const SmemLevel<T> &C, int sweeps)
{
    TSmooth<T, kWarp>(C, 0, true);
    TSmooth<T, kWarp>(C, 1, false);
    for (int s = 1; s < sweeps; s++)
    {
        TSmooth<T, kWarp>(C, 0, false);
        TSmooth<T, kWarp>(C, 1, false);
    }
    for (int s = 0; s < sweeps; s++)
    {
        TSmooth<T, kWarp>(C, 1, false);
        TSmooth<T, kWarp>(C, 0, false);
    }
}

// The ascent into level l: the prolonged correction, then the post-sweeps black first.
template <typename T, bool kWarp> __device__ void TUp(const SmemLevel<T> &F, const SmemLevel<T> &C, int post)
{
    TProlong<T, kWarp>(F, C);
    for (int s = 0; s < post; s++)
    {
        TSmooth<T, kWarp>(F, 1, false);
        TSmooth<T, kWarp>(F, 0, false);
    }
}

template <typename T> __device__ __forceinline__ void TailBody(const TailArgs<T> &A)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double sInv[kMaxTailLevels][32];
    __shared__ int sCount[kMaxTailLevels][2];
    // stage: cell types, codes and lists of every tail level, zero corrections and residuals, the first level's r
    for (int l = 0; l < A.nlev; l++)
    {
        const LevelView &g = A.lv[l].v;
        const SmemLevel<T> S = Bind<T>(A.lv[l], smem);
        const unsigned *gl = A.lists + A.lv[l].listOff;
        for (long long c = threadIdx.x; c < g.cells; c += blockDim.x)
        {
            ((uint8_t *)S.v.code)[c] = g.code[c];
            ((uint8_t *)S.v.types)[c] = g.types[c];
            S.e[c] = (T)0;
            S.res[c] = (T)0;
            S.r[c] = l == 0 ? A.rIn[c] : (T)0;
            S.list[c] = gl[c];
        }
        if (threadIdx.x < 32)
            sInv[l][threadIdx.x] = threadIdx.x ? 1.0 / (0.5 * g.gamma * (double)threadIdx.x) : 0.0;
        if (threadIdx.x < 2) sCount[l][threadIdx.x] = A.counts[2 * l + threadIdx.x];
    }
    __syncthreads();
    // the diagonal half-units of the uniform levels' unknowns: 2 per FLUID neighbour, 2 per interior Dirichlet
    // neighbour, 4 per Dirichlet ring neighbour (ring factor 2)
    for (int l = 0; l < A.nlev; l++)
    {
        const SmemLevel<T> S = Bind<T>(A.lv[l], smem);
        const LevelView &v = S.v;
        if (v.stretched) continue;
        const int nq = v.dim == 3 ? 6 : 4;
        for (long long c = threadIdx.x; c < v.cells; c += blockDim.x)
        {
            const unsigned code = v.code[c];
            unsigned units = 0;
            if (code & CODE_UNKNOWN)
            {
                units = 2u * (unsigned)__popc(code & CODE_FLUID_MASK);
                if (code & CODE_DIRICHLET)
                {
                    int i, j, k;
                    Decode(v, c, i, j, k);
                    for (int q = 0; q < nq; q++)
                        if (IsDirichlet(v.types[c + NbrOffset(v, q)]))
                        {
                            const int ni = i + (q == 0) - (q == 1), nj = j + (q == 2) - (q == 3),
                                      nk = k + (q == 4) - (q == 5);
                            units += OnRing(v, ni, nj, nk) ? 4u : 2u;
                        }
                }
                units |= 0x80u;
            }
            S.du[c] = (uint8_t)units;
        }
    }
    __syncthreads();
    auto lev = [&](int l) {
        SmemLevel<T> s = Bind<T>(A.lv[l], smem);
        s.nRed = sCount[l][0];
        s.nBlack = sCount[l][1];
        s.inv = sInv[l];
        return s;
    };
    const int last = A.nlev - 1;
    // wl: the first level from which every coarser one has at most 32 unknowns of each colour (warp 0 runs those)
    int wl = A.nlev;
    for (int l = last; l >= 0 && sCount[l][0] <= 32 && sCount[l][1] <= 32; l--) wl = l;
    const int top = wl < last ? wl : last;
    for (int l = 0; l < top; l++) TDown<T, false>(lev(l), lev(l + 1), A.pre);
    if (wl > last) TCoarsest<T, false>(lev(last), A.coarseSweeps);
    else
    {
        if (threadIdx.x < 32)
        {
            for (int l = wl; l < last; l++) TDown<T, true>(lev(l), lev(l + 1), A.pre);
            TCoarsest<T, true>(lev(last), A.coarseSweeps);
            for (int l = last - 1; l >= wl; l--) TUp<T, true>(lev(l), lev(l + 1), A.post);
        }
        __syncthreads();
    }
    for (int l = top - 1; l >= 0; l--) TUp<T, false>(lev(l), lev(l + 1), A.post);
    const SmemLevel<T> F0 = Bind<T>(A.lv[0], smem);
    for (long long c = threadIdx.x; c < A.lv[0].v.cells; c += blockDim.x) A.eOut[c] = F0.e[c];
}

template <typename T> __global__ void __launch_bounds__(kTailThreads) k_tail(TailArgs<T> A)
{
    PdlWait();
    PdlTrigger();
    TailBody<T>(A);
}

// batched (nb_batch.cu): block z runs the coarse end of the request at list[z], its arguments copied from global
// memory into shared memory first
__global__ void __launch_bounds__(kTailThreads) kb_tail(const BatchReq *__restrict__ rq, BatchList a)
{
    PdlWait();
    PdlTrigger();
    const int q = BatchReqOf(a);
    if (q < 0) return;
    __shared__ TailArgs<float> sA;
    const TailArgs<float> *g = static_cast<const TailArgs<float> *>(rq[q].tail);
    {
        const int n = (int)(sizeof(TailArgs<float>) / sizeof(int));
        const int *src = reinterpret_cast<const int *>(g);
        int *dst = reinterpret_cast<int *>(&sA);
        for (int t = threadIdx.x; t < n; t += blockDim.x) dst[t] = src[t];
    }
    __syncthreads();
    TailBody<float>(sA);
}

// The per-colour lists of every tail level's unknowns, once per layout: entries packed (i << 20 | j << 10 | k), red
// ones from the front of the level's segment, black ones from the back; their order within a colour does not matter
// (the cells of one colour are updated independently).
__global__ void __launch_bounds__(1024) k_tail_lists(TailArgs<float> A)
{
    __shared__ int cnt[kMaxTailLevels][2];
    if (threadIdx.x < 2 * kMaxTailLevels) cnt[threadIdx.x >> 1][threadIdx.x & 1] = 0;
    __syncthreads();
    for (int l = 0; l < A.nlev; l++)
    {
        const LevelView &g = A.lv[l].v;
        unsigned *list = const_cast<unsigned *>(A.lists) + A.lv[l].listOff;
        for (long long c = threadIdx.x; c < g.cells; c += blockDim.x)
        {
            if (!(g.code[c] & CODE_UNKNOWN)) continue;
            int i, j, k;
            Decode(g, c, i, j, k);
            const int col = (i + j + k) & 1;
            const int pos = atomicAdd(&cnt[l][col], 1);
            const unsigned packed = ((unsigned)i << 20) | ((unsigned)j << 10) | (unsigned)k;
            if (col == 0) list[pos] = packed;
            else list[g.cells - 1 - pos] = packed;
        }
    }
    __syncthreads();
    if (threadIdx.x < 2 * A.nlev) const_cast<int *>(A.counts)[threadIdx.x] = cnt[threadIdx.x >> 1][threadIdx.x & 1];
}

long long TailListEntries(const LevelView *levels, int nlev)
{
    long long n = 0;
    for (int l = 0; l < nlev; l++) n += levels[l].cells;
    return n;
}

void LaunchTailLists(const LevelView *levels, int nlev, unsigned *lists, int *counts, cudaStream_t st)
{
    TailArgs<float> A{};
    unsigned off = 0;
    for (int l = 0; l < nlev; l++)
    {
        A.lv[l].v = levels[l];
        A.lv[l].listOff = off;
        off += (unsigned)levels[l].cells;
    }
    A.nlev = nlev;
    A.lists = lists;
    A.counts = counts;
    NB_COUNT_LAUNCH();
    k_tail_lists<<<1, 1024, 0, st>>>(A);
}

template <typename T> size_t TailSmemBytes(const LevelView *levels, int nlev)
{
    size_t bytes = 0;
    for (int l = 0; l < nlev; l++) bytes += LevelBytes<T>(levels[l].cells);
    return bytes;
}

template <typename T> static bool PrepareTailOnce()
{
    if (sizeof(T) == 4 &&
        cudaFuncSetAttribute(kb_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTailMaxSmem) != cudaSuccess)
        return false;
    return cudaFuncSetAttribute(k_tail<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTailMaxSmem) ==
           cudaSuccess;
}

// Once per device and precision: changing a kernel's attribute on every layout change would take the driver's
// locks under a server's running solves.
template <typename T> bool PrepareTail(size_t bytes)
{
    if (bytes > kTailMaxSmem) return false;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    static std::mutex mu;
    static std::set<int> done;
    std::lock_guard<std::mutex> lock(mu);
    const int key = 2 * dev + (sizeof(T) == 4 ? 0 : 1);
    if (done.count(key)) return true;
    if (!PrepareTailOnce<T>()) return false;
    done.insert(key);
    return true;
}
// The coarse end's arguments of one request (FP32), for a batch's table in device memory: *bytes = their size,
// and when out is not null they are written there; *smem = the dynamic shared memory of its launch.
void TailArgsFor(const LevelView *levels, int nlev, const float *rIn, float *eOut, int pre, int post,
                 int coarseSweeps, const unsigned *lists, const int *counts, void *out, size_t *bytes, size_t *smem)
{
    TailArgs<float> A{};
    unsigned off = 0, listOff = 0;
    for (int l = 0; l < nlev; l++)
    {
        A.lv[l].v = levels[l];
        A.lv[l].off = off;
        A.lv[l].listOff = listOff;
        off += LevelBytes<float>(levels[l].cells);
        listOff += (unsigned)levels[l].cells;
    }
    A.nlev = nlev;
    A.rIn = rIn;
    A.eOut = eOut;
    A.pre = pre < 1 ? 1 : pre;
    A.post = post < 1 ? 1 : post;
    A.coarseSweeps = coarseSweeps < 1 ? 1 : coarseSweeps;
    A.lists = lists;
    A.counts = counts;
    *bytes = sizeof(A);
    *smem = off;
    if (out) std::memcpy(out, &A, sizeof(A));
}

void LaunchBatchTail(const BatchReq *rq, BatchList a, int cap, size_t smem, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    LaunchPdl(kb_tail, dim3(1, 1, cap), dim3(kTailThreads), smem, st, rq, a);
}

template <typename T>
void LaunchTail(const LevelView *levels, int nlev, const T *rIn, T *eOut, int pre, int post, int coarseSweeps,
                const unsigned *lists, const int *counts, cudaStream_t st)
{
    TailArgs<T> A{};
    unsigned off = 0, listOff = 0;
    for (int l = 0; l < nlev; l++)
    {
        A.lv[l].v = levels[l];
        A.lv[l].off = off;
        A.lv[l].listOff = listOff;
        off += LevelBytes<T>(levels[l].cells);
        listOff += (unsigned)levels[l].cells;
    }
    A.nlev = nlev;
    A.rIn = rIn;
    A.eOut = eOut;
    A.pre = pre < 1 ? 1 : pre;
    A.post = post < 1 ? 1 : post;
    A.coarseSweeps = coarseSweeps < 1 ? 1 : coarseSweeps;
    A.lists = lists;
    A.counts = counts;
    NB_COUNT_LAUNCH();
    LaunchPdl(k_tail<T>, dim3(1), dim3(kTailThreads), (size_t)off, st, A);
}

template size_t TailSmemBytes<float>(const LevelView *, int);
template size_t TailSmemBytes<double>(const LevelView *, int);
template bool PrepareTail<float>(size_t);
template bool PrepareTail<double>(size_t);
template void LaunchTail<float>(const LevelView *, int, const float *, float *, int, int, int, const unsigned *,
                                const int *, cudaStream_t);
template void LaunchTail<double>(const LevelView *, int, const double *, double *, int, int, int, const unsigned *,
                                 const int *, cudaStream_t);

} // namespace nb
