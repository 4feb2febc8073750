// The coarse end of the multigrid V-cycle in one thread block: every level from `tailStart` down (at most a few
// thousand cells each, about 16^3 and below) lives in shared memory, and the block runs their pre-smoothing,
// residual, restriction, coarsest sweeps, prolongation and post-smoothing back to back with __syncthreads between
// the phases. It reads the restricted residual of the first tail level from global memory and writes that level's
// correction back; the finer levels' kernels on either side are unchanged. The operations are the ones of
// nb_kernels.cu (same stencil, transfers and colour order), so the V-cycle stays the same symmetric operator.
#include "nb_kernels.h"

namespace nb
{

template <typename T> struct TailLevel
{
    LevelView v;
    unsigned off; // byte offset of the level's arrays in shared memory
};

template <typename T> struct TailArgs
{
    TailLevel<T> lv[kMaxTailLevels];
    int nlev;
    const T *rIn; // residual of the first tail level (global)
    T *eOut;      // its correction (global)
    int pre, post, coarseSweeps;
};

// The level's arrays in shared memory: r, e, res (T), then code and types (bytes), then the list of its unknowns
// (4 bytes each: red ones from the front, black ones from the back), each padded to 16 bytes.
template <typename T> __host__ __device__ inline unsigned LevelBytes(long long cells)
{
    const unsigned a = (unsigned)((cells * sizeof(T) + 15) / 16 * 16);
    const unsigned b = (unsigned)((cells + 15) / 16 * 16);
    const unsigned l = (unsigned)((cells * 4 + 15) / 16 * 16);
    return 3 * a + 2 * b + l;
}

template <typename T> struct SmemLevel
{
    LevelView v; // types/code point into shared memory
    T *r, *e, *res;
    unsigned *list; // packed (i << 20 | j << 10 | k) of the unknowns; red [0, nRed), black [cells - nBlack, cells)
    int nRed, nBlack;
};

// unknowns per colour of each tail level, counted while the lists are built
__shared__ int g_tailCount[kMaxTailLevels][2];

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
    s.list = (unsigned *)(base + 3 * a + 2 * b);
    return s;
}

// the level bound with its unknown counts (valid once the lists are built)
template <typename T> __device__ __forceinline__ SmemLevel<T> BindL(const TailLevel<T> &tl, unsigned char *smem, int l)
{
    SmemLevel<T> s = Bind<T>(tl, smem);
    s.nRed = g_tailCount[l][0];
    s.nBlack = g_tailCount[l][1];
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

template <typename T> __device__ void TSmooth(const SmemLevel<T> &L, int colour, bool first)
{
    const LevelView &v = L.v;
    const int n = ListLen(L, colour);
    for (int t = threadIdx.x; t < n; t += blockDim.x)
    {
        int i, j, k;
        Unpack(ListAt(L, colour, t), i, j, k);
        const long long c = (long long)i * v.sI + (long long)j * v.sJ + k;
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
    __syncthreads();
}

template <typename T> __device__ void TResidual(const SmemLevel<T> &L)
{
    const LevelView &v = L.v;
    const int n = ListLen(L, 2);
    for (int t = threadIdx.x; t < n; t += blockDim.x)
    {
        int i, j, k;
        Unpack(ListAt(L, 2, t), i, j, k);
        const long long c = (long long)i * v.sI + (long long)j * v.sJ + k;
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
    __syncthreads();
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

template <typename T> __device__ void TRestrict(const SmemLevel<T> &F, const SmemLevel<T> &C)
{
    const LevelView &fv = F.v, &cv = C.v;
    const int n = ListLen(C, 2);
    for (int t = threadIdx.x; t < n; t += blockDim.x)
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
    __syncthreads();
}

template <typename T> __device__ void TProlong(const SmemLevel<T> &F, const SmemLevel<T> &C)
{
    const LevelView &fv = F.v, &cv = C.v;
    const int n = ListLen(F, 2);
    for (int t = threadIdx.x; t < n; t += blockDim.x)
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
    __syncthreads();
}

template <typename T> __global__ void __launch_bounds__(1024) k_tail(TailArgs<T> A)
{
    extern __shared__ __align__(16) unsigned char smem[];
    // stage: cell types and codes of every tail level, zero corrections and residuals, the first level's r
    for (int l = 0; l < A.nlev; l++)
    {
        const LevelView &g = A.lv[l].v;
        const SmemLevel<T> S = Bind<T>(A.lv[l], smem);
        for (long long c = threadIdx.x; c < g.cells; c += blockDim.x)
        {
            ((uint8_t *)S.v.code)[c] = g.code[c];
            ((uint8_t *)S.v.types)[c] = g.types[c];
            S.e[c] = (T)0;
            S.res[c] = (T)0;
            S.r[c] = l == 0 ? A.rIn[c] : (T)0;
        }
    }
    if (threadIdx.x < 2 * kMaxTailLevels) g_tailCount[threadIdx.x >> 1][threadIdx.x & 1] = 0;
    __syncthreads();
    // the unknowns of every level by colour (i + j + k) & 1; their order within a colour does not matter (the
    // cells of one colour are updated independently)
    for (int l = 0; l < A.nlev; l++)
    {
        const LevelView &g = A.lv[l].v;
        const SmemLevel<T> S = Bind<T>(A.lv[l], smem);
        for (long long c = threadIdx.x; c < g.cells; c += blockDim.x)
        {
            if (!(S.v.code[c] & CODE_UNKNOWN)) continue;
            int i, j, k;
            Decode(g, c, i, j, k);
            const int col = (i + j + k) & 1;
            const int pos = atomicAdd(&g_tailCount[l][col], 1);
            const unsigned packed = ((unsigned)i << 20) | ((unsigned)j << 10) | (unsigned)k;
            if (col == 0) S.list[pos] = packed;
            else S.list[g.cells - 1 - pos] = packed;
        }
    }
    __syncthreads();
    const int last = A.nlev - 1;
    for (int l = 0; l < last; l++)
    {
        const SmemLevel<T> F = BindL<T>(A.lv[l], smem, l);
        TSmooth<T>(F, 0, true);
        TSmooth<T>(F, 1, false);
        for (int s = 1; s < A.pre; s++)
        {
            TSmooth<T>(F, 0, false);
            TSmooth<T>(F, 1, false);
        }
        TResidual<T>(F);
        TRestrict<T>(F, BindL<T>(A.lv[l + 1], smem, l + 1));
    }
    {
        const SmemLevel<T> C = BindL<T>(A.lv[last], smem, last);
        TSmooth<T>(C, 0, true);
        TSmooth<T>(C, 1, false);
        for (int s = 1; s < A.coarseSweeps; s++)
        {
            TSmooth<T>(C, 0, false);
            TSmooth<T>(C, 1, false);
        }
        for (int s = 0; s < A.coarseSweeps; s++)
        {
            TSmooth<T>(C, 1, false);
            TSmooth<T>(C, 0, false);
        }
    }
    for (int l = last - 1; l >= 0; l--)
    {
        const SmemLevel<T> F = BindL<T>(A.lv[l], smem, l);
        TProlong<T>(F, BindL<T>(A.lv[l + 1], smem, l + 1));
        for (int s = 0; s < A.post; s++)
        {
            TSmooth<T>(F, 1, false);
            TSmooth<T>(F, 0, false);
        }
    }
    const SmemLevel<T> F0 = Bind<T>(A.lv[0], smem);
    for (long long c = threadIdx.x; c < A.lv[0].v.cells; c += blockDim.x) A.eOut[c] = F0.e[c];
}

template <typename T> size_t TailSmemBytes(const LevelView *levels, int nlev)
{
    size_t bytes = 0;
    for (int l = 0; l < nlev; l++) bytes += LevelBytes<T>(levels[l].cells);
    return bytes;
}

template <typename T> bool PrepareTail(size_t bytes)
{
    if (bytes > kTailMaxSmem) return false;
    return cudaFuncSetAttribute(k_tail<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTailMaxSmem) ==
           cudaSuccess;
}

template <typename T>
void LaunchTail(const LevelView *levels, int nlev, const T *rIn, T *eOut, int pre, int post, int coarseSweeps,
                cudaStream_t st)
{
    TailArgs<T> A{};
    unsigned off = 0;
    for (int l = 0; l < nlev; l++)
    {
        A.lv[l].v = levels[l];
        A.lv[l].off = off;
        off += LevelBytes<T>(levels[l].cells);
    }
    A.nlev = nlev;
    A.rIn = rIn;
    A.eOut = eOut;
    A.pre = pre < 1 ? 1 : pre;
    A.post = post < 1 ? 1 : post;
    A.coarseSweeps = coarseSweeps < 1 ? 1 : coarseSweeps;
    NB_COUNT_LAUNCH();
    k_tail<T><<<1, 1024, off, st>>>(A);
}

template size_t TailSmemBytes<float>(const LevelView *, int);
template size_t TailSmemBytes<double>(const LevelView *, int);
template bool PrepareTail<float>(size_t);
template bool PrepareTail<double>(size_t);
template void LaunchTail<float>(const LevelView *, int, const float *, float *, int, int, int, cudaStream_t);
template void LaunchTail<double>(const LevelView *, int, const double *, double *, int, int, int, cudaStream_t);

} // namespace nb
