// One full red-black Gauss-Seidel sweep per launch, for 3D levels: the block stages (fast x mid) tiles of the
// iterate, the right-hand side and the cell codes in shared memory and marches along the slow axis, updating the
// first colour on the tile plus a one-cell halo (the halo values are recomputed by the neighbouring blocks too,
// identically) and then the second colour on the tile, one plane behind. Every plane of e, r and the codes is read
// from global memory once and the result written once, instead of two full passes per sweep.
//
// Variants (template flags):
//   kFirst   -- the sweep starts from a zero iterate (the pre-smoothing of a V-cycle): no iterate is read;
//   kProlong -- the iterate is e + P(e_coarse), the coarse-grid correction applied on the fly (the post-smoothing);
//   kDot     -- the block also sums r.z, z and r of the final values (the r.z of CG, fused into the V-cycle's end).
// The sweep reads e_in and writes e_out (different arrays), so no block reads a value another block has updated.
#include "nb_kernels.h"

namespace nb
{

constexpr int kFT = 64, kMT = 8;               // tile: 64 cells along the fast axis, 8 along the mid axis
constexpr int kH2F = kFT + 4, kH2M = kMT + 4;  // tile with a two-cell halo: where the iterate is needed
constexpr int kH1F = kFT + 2, kH1M = kMT + 2;  // tile with a one-cell halo: where the first colour is updated
constexpr int kH2 = kH2F * kH2M, kH1 = kH1F * kH1M, kT = kFT * kMT;
constexpr int kSweepThreads = 256;

template <typename T> struct SweepSmem
{
    T eold[3][kH2];   // iterate, planes p, p+1, p+2 (rolling)
    T rn[3][kH1];     // after the first colour, planes p-1, p, p+1 (rolling)
    T r[2][kH1];      // right-hand side, planes p, p+1 (rolling)
    uint8_t code[3][kH2];
};

// prolongation of the coarse correction at fine cell (a, b, d) (nb_kernels.cu k_prolong, same weights)
template <typename T>
__device__ __forceinline__ T ProlongAt(const LevelView &cv, const T *__restrict__ ec, int a, int b, int d)
{
    const int A = (a + 1) >> 1, B = (b + 1) >> 1, D = (d + 1) >> 1;
    const int si = (a & 1) ? -1 : 1, sj = (b & 1) ? -1 : 1, sk = (d & 1) ? -1 : 1;
    const T wv[2] = {(T)0.75, (T)0.25};
    const long long parent = (long long)A * cv.sI + (long long)B * cv.sJ + D;
    T acc = (T)0, extra = (T)0;
#pragma unroll
    for (int di = 0; di < 2; di++)
#pragma unroll
        for (int dj = 0; dj < 2; dj++)
#pragma unroll
            for (int dk = 0; dk < 2; dk++)
            {
                const long long cc = parent + (long long)(di * si) * cv.sI + (long long)(dj * sj) * cv.sJ + dk * sk;
                const T w = wv[di] * wv[dj] * wv[dk];
                if ((di | dj | dk) && cv.types[cc] == SOLID) extra += w;
                else acc += w * ec[cc];
            }
    return acc + extra * ec[parent];
}

template <typename T, bool kFirst, bool kProlong, bool kDot>
__global__ void __launch_bounds__(kSweepThreads) k_rb_sweep(LevelView v, LevelView cv, const T *__restrict__ r,
                                                            const T *__restrict__ eIn, const T *__restrict__ ec,
                                                            T *__restrict__ eOut, int firstColour, int chunk,
                                                            Reducer R, const int *it, int baseEven, int baseOdd)
{
    extern __shared__ __align__(16) unsigned char smemRaw[];
    SweepSmem<T> &S = *reinterpret_cast<SweepSmem<T> *>(smemRaw);
    const int tid = threadIdx.x;
    // interior origin of the tile: k (fast) and j (mid); planes i (slow) in [pb, pe)
    const int k0 = 1 + blockIdx.x * kFT, j0 = 1 + blockIdx.y * kMT;
    const int pb = 1 + blockIdx.z * chunk, pe = min(pb + chunk, v.Ny - 1);
    const int Nx = v.Nx, Ny = v.Ny, Nz = v.Nz;
    const long long sI = v.sI, sJ = v.sJ;
    double acc[3] = {0.0, 0.0, 0.0};

    for (int q = pb - 4; q < pe; q++)
    {
        // ---- stage plane q+2 of the iterate and codes (two-cell halo), plane q+1 of r (one-cell halo) ----
        {
            const int i = q + 2, slotE = (i + 3) % 3;
            const bool planeIn = i >= 0 && i <= Ny - 1;
            for (int t = tid; t < kH2; t += kSweepThreads)
            {
                const int a = t / kH2F, b = t - a * kH2F;
                const int j = j0 - 2 + a, k = k0 - 2 + b;
                T val = (T)0;
                uint8_t cd = 0;
                if (planeIn && j >= 0 && j <= Nx - 1 && k >= 0 && k <= Nz - 1)
                {
                    const long long c = (long long)i * sI + (long long)j * sJ + k;
                    cd = v.code[c];
                    if (!kFirst)
                    {
                        val = eIn[c];
                        if (kProlong && (cd & CODE_UNKNOWN)) val += ProlongAt<T>(cv, ec, i, j, k);
                    }
                }
                S.eold[slotE][t] = val;
                S.code[slotE][t] = cd;
            }
            const int ir = q + 1, slotR = (ir + 2) % 2;
            const bool planeR = ir >= 0 && ir <= Ny - 1;
            for (int t = tid; t < kH1; t += kSweepThreads)
            {
                const int a = t / kH1F, b = t - a * kH1F;
                const int j = j0 - 1 + a, k = k0 - 1 + b;
                T val = (T)0;
                if (planeR && j >= 0 && j <= Nx - 1 && k >= 0 && k <= Nz - 1)
                    val = r[(long long)ir * sI + (long long)j * sJ + k];
                S.r[slotR][t] = val;
            }
        }
        __syncthreads();
        // ---- first colour on plane q+1 over the tile + one-cell halo ----
        if (q + 1 >= pb - 1)
        {
            const int i = q + 1;
            const int sm = (i + 2) % 3, s0 = (i + 3) % 3, sp = (i + 4) % 3; // planes i-1, i, i+1 of eold
            const int sr = (i + 3) % 3, srr = (i + 2) % 2;
            for (int t = tid; t < kH1; t += kSweepThreads)
            {
                const int a = t / kH1F, b = t - a * kH1F;
                const int h = (a + 1) * kH2F + (b + 1); // index in the two-cell-halo tile
                const int j = j0 - 1 + a, k = k0 - 1 + b;
                const unsigned cd = S.code[s0][h];
                T val = S.eold[s0][h];
                if ((cd & CODE_UNKNOWN) && ((i + j + k) & 1) == firstColour)
                {
                    T cq[6], diag;
                    CodeStencil<T>(v, i, j, k, (long long)i * sI + (long long)j * sJ + k, cd, cq, diag);
                    T rhs = S.r[srr][t];
                    if (!kFirst)
                    {
                        if (cd & 1u) rhs += cq[0] * S.eold[sp][h];
                        if (cd & 2u) rhs += cq[1] * S.eold[sm][h];
                        if (cd & 4u) rhs += cq[2] * S.eold[s0][h + kH2F];
                        if (cd & 8u) rhs += cq[3] * S.eold[s0][h - kH2F];
                        if (cd & 16u) rhs += cq[4] * S.eold[s0][h + 1];
                        if (cd & 32u) rhs += cq[5] * S.eold[s0][h - 1];
                    }
                    val = diag != (T)0 ? rhs / diag : (T)0;
                }
                S.rn[sr][t] = val;
            }
        }
        __syncthreads();
        // ---- second colour on plane q over the tile; write the plane ----
        if (q >= pb)
        {
            const int i = q;
            const int sm = (i + 2) % 3, s0 = (i + 3) % 3, sp = (i + 4) % 3; // planes i-1, i, i+1 of rn
            const int sc = (i + 3) % 3, srr = (i + 2) % 2;
            for (int t = tid; t < kT; t += kSweepThreads)
            {
                const int a = t / kFT, b = t - a * kFT;
                const int j = j0 + a, k = k0 + b;
                if (j > Nx - 2 || k > Nz - 2) continue;
                const int h1 = (a + 1) * kH1F + (b + 1);
                const int h2 = (a + 2) * kH2F + (b + 2);
                const unsigned cd = S.code[sc][h2];
                T val = S.rn[s0][h1];
                const T rv = S.r[srr][h1];
                if ((cd & CODE_UNKNOWN) && ((i + j + k) & 1) != firstColour)
                {
                    T cq[6], diag;
                    CodeStencil<T>(v, i, j, k, (long long)i * sI + (long long)j * sJ + k, cd, cq, diag);
                    T rhs = rv;
                    if (cd & 1u) rhs += cq[0] * S.rn[sp][h1];
                    if (cd & 2u) rhs += cq[1] * S.rn[sm][h1];
                    if (cd & 4u) rhs += cq[2] * S.rn[s0][h1 + kH1F];
                    if (cd & 8u) rhs += cq[3] * S.rn[s0][h1 - kH1F];
                    if (cd & 16u) rhs += cq[4] * S.rn[s0][h1 + 1];
                    if (cd & 32u) rhs += cq[5] * S.rn[s0][h1 - 1];
                    val = diag != (T)0 ? rhs / diag : (T)0;
                }
                eOut[(long long)i * sI + (long long)j * sJ + k] = val;
                if (kDot && (cd & CODE_UNKNOWN))
                {
                    acc[0] += (double)rv * (double)val;
                    acc[1] += (double)val;
                    acc[2] += (double)rv;
                }
            }
        }
        __syncthreads();
    }
    if (kDot) GridReduce<3>(R, acc, (*it & 1) ? baseOdd : baseEven);
}

template <typename T> static size_t SweepSmemBytes() { return sizeof(SweepSmem<T>); }

template <typename T, bool kFirst, bool kProlong, bool kDot> static void SetSweepAttr()
{
    cudaFuncSetAttribute(k_rb_sweep<T, kFirst, kProlong, kDot>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)SweepSmemBytes<T>());
}

template <typename T> void PrepareSweeps()
{
    SetSweepAttr<T, true, false, false>();
    SetSweepAttr<T, true, false, true>();
    SetSweepAttr<T, false, false, false>();
    SetSweepAttr<T, false, true, false>();
    SetSweepAttr<T, false, true, true>();
    SetSweepAttr<T, false, false, true>();
}

// planes per block: enough that the four planes of lead-in are a small share, few enough to fill the SMs
static inline int SweepChunk(const LevelView &v)
{
    const long long tiles = (long long)((v.fastLen + kFT - 1) / kFT) * ((v.midLen + kMT - 1) / kMT);
    int chunk = 16;
    while (chunk > 4 && tiles * ((v.slowLen + chunk - 1) / chunk) < 148 * 4) chunk /= 2;
    return chunk;
}

template <typename T>
void LaunchRBSweep(const LevelView &v, const LevelView &cv, const T *r, const T *eIn, const T *ec, T *eOut,
                   int firstColour, bool first, bool prolong, bool dot, const Reducer &R, const int *it, int baseEven,
                   int baseOdd, cudaStream_t st)
{
    const int chunk = SweepChunk(v);
    dim3 grid((unsigned)((v.fastLen + kFT - 1) / kFT), (unsigned)((v.midLen + kMT - 1) / kMT),
              (unsigned)((v.slowLen + chunk - 1) / chunk));
    const size_t smem = SweepSmemBytes<T>();
    NB_COUNT_LAUNCH();
#define NB_SWEEP(F, P, D)                                                                                          \
    k_rb_sweep<T, F, P, D><<<grid, kSweepThreads, smem, st>>>(v, cv, r, eIn, ec, eOut, firstColour, chunk, R, it,     \
                                                              baseEven, baseOdd)
    if (first)
    {
        if (dot) NB_SWEEP(true, false, true);
        else NB_SWEEP(true, false, false);
    }
    else if (prolong)
    {
        if (dot) NB_SWEEP(false, true, true);
        else NB_SWEEP(false, true, false);
    }
    else
    {
        if (dot) NB_SWEEP(false, false, true);
        else NB_SWEEP(false, false, false);
    }
#undef NB_SWEEP
}

template void PrepareSweeps<float>();
template void PrepareSweeps<double>();
template void LaunchRBSweep<float>(const LevelView &, const LevelView &, const float *, const float *, const float *,
                                   float *, int, bool, bool, bool, const Reducer &, const int *, int, int,
                                   cudaStream_t);
template void LaunchRBSweep<double>(const LevelView &, const LevelView &, const double *, const double *,
                                    const double *, double *, int, bool, bool, bool, const Reducer &, const int *, int,
                                    int, cudaStream_t);

} // namespace nb
