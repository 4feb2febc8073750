// Multigrid and PCG kernels for 3D levels of a uniform grid in FP32 (the inner solve of the mixed-precision form),
// built for memory throughput.
//
// Cell pairs. With Nz even, the two cells (i, j, 2m) and (i, j, 2m+1) form an 8-byte aligned pair, and a plane of
// Nx*Nz cells is Nx*Nz/2 consecutive pairs. Thread t of the launch takes pair t of the plane (crossing row ends
// freely: a row's ring cells ride along, their vector entries are zero) and marches along i over up to kPairS
// planes (fewer on small levels, so that a launch still has about 148 x 8 blocks and no long serial chains),
// keeping the pairs of planes i-1, i, i+1 in registers. A warp's load of one plane is 256 contiguous bytes; the j
// neighbours are the pairs Nz/2 away; the k neighbours are the other cell of the pair and, across the pair
// boundary, the neighbouring lane's pair (a shuffle; lanes 0 and 31 load that one cell).
//
// Unmasked stencil. Every vector is zero off the unknowns (interior FLUID cells), so sum_q c_q x_q over the FLUID
// neighbours equals gamma times the plain sum of all six neighbours on a uniform level. What remains per cell is
// the diagonal, which on a uniform level is gamma/2 times an integer: 2 per FLUID neighbour, 2 per interior
// Dirichlet neighbour, 4 per Dirichlet ring neighbour (ring factor FaceGap/(Width/2) = 2,
// PressureSettings.h:307-310). It is kept per cell in one byte, `du` = 0x80 | half-units for an unknown, 0 elsewhere,
// and divided through a 32-entry reciprocal table in shared memory (entry 0 is 0, which leaves non-unknowns and
// isolated cells at zero like the reference's zero diagonal guard).
#include "nb_kernels.h"

#include <algorithm>

namespace nb
{

namespace
{

__device__ __forceinline__ float2 Ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ unsigned LdDu(const uint8_t *p) { return *reinterpret_cast<const unsigned short *>(p); }

// 1 / (gamma/2 * units), entry 0 = 0
__device__ __forceinline__ void FillInverse(float *inv, double gamma)
{
    if (threadIdx.x < 32) inv[threadIdx.x] = threadIdx.x ? 1.0f / (0.5f * (float)gamma * (float)threadIdx.x) : 0.0f;
    __syncthreads();
}

__device__ __forceinline__ float Unk(unsigned du) { return (du & 0x80u) ? 1.0f : 0.0f; }

} // namespace

// ---------------------------------------------------------------------------------------------------------------
// diagonal units
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_build_du(LevelView v, uint8_t *du)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < v.cells;
         c += (long long)gridDim.x * blockDim.x)
    {
        const int k = (int)(c % v.Nz);
        const long long rr = c / v.Nz;
        const int j = (int)(rr % v.Nx), i = (int)(rr / v.Nx);
        const bool interior = i > 0 && i < v.Ny - 1 && j > 0 && j < v.Nx - 1 && k > 0 && k < v.Nz - 1;
        const long long o = VecIdx(v, i, j, k); // the grid layout, or the colour-split one of a split level
        if (!interior || v.types[c] != FLUID) { du[o] = 0; continue; }
        unsigned units = 0;
        for (int q = 0; q < 6; q++)
        {
            const int t = v.types[c + NbrOffset(v, q)];
            if (t == FLUID) units += 2;
            else if (IsDirichlet(t))
            {
                const int ni = i + (q == 0) - (q == 1), nj = j + (q == 2) - (q == 3), nk = k + (q == 4) - (q == 5);
                units += OnRing(v, ni, nj, nk) ? 4 : 2;
            }
        }
        du[o] = (uint8_t)(0x80u | units);
    }
}

bool PairLevelShape(const LevelView &v) { return v.dim == 3 && (v.Nz % 2) == 0 && v.Ny >= 3; }

void LaunchBuildDu(const LevelView &v, uint8_t *du, cudaStream_t st)
{
    int blocks = (int)((v.cells + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    NB_COUNT_LAUNCH();
    k_build_du<<<blocks, 256, 0, st>>>(v, du);
}

// planes per thread at least in the launches that end in a grid-wide sum: fewer blocks, fewer partial sums for the
// last block to add (measured: 16 beats the 8 of the plain sweeps there)
constexpr int kReduceS = 16;

// ---------------------------------------------------------------------------------------------------------------
// smoothing
// ---------------------------------------------------------------------------------------------------------------

// The first red-black sweep from a zero iterate: red e = r / diag, then black e = (r + gamma * sum of the red
// neighbours) / diag, with the red neighbours formed on the fly from r and du. Colour = (i + j + k) & 1, red = 0.
__global__ void __launch_bounds__(kPairThreads) k_pair_first(LevelView v, const uint8_t *__restrict__ du,
                                                             const float *__restrict__ r, float *__restrict__ e)
{
    __shared__ float inv[32];
    FillInverse(inv, v.gamma);
    const PairPos P = PairStart(v);
    const float g = (float)v.gamma;
    const float *rp = r + P.base;
    const uint8_t *dp = du + P.base;
    float *ep = e + P.base;
    // red-only pair of a plane: red cells carry r/diag, black cells 0
    auto red = [&](float2 rv, unsigned d, int i) {
        const int c0 = (i + P.j + P.k0) & 1; // colour of the first cell
        const float a = rv.x * inv[d & 0x7Fu], b = rv.y * inv[(d >> 8) & 0x7Fu];
        return c0 == 0 ? make_float2(a, 0.f) : make_float2(0.f, b);
    };
    const int o0 = -P.sI;
    float2 RM = red(Ld2(rp + o0), LdDu(dp + o0), P.i0 - 1);
    float2 rC = Ld2(rp);
    unsigned dC = LdDu(dp);
    float2 RC = red(rC, dC, P.i0);
    int off = 0;
    for (int i = P.i0; i < P.i1; i++, off += P.sI)
    {
        const float2 rP = Ld2(rp + off + P.sI);
        const unsigned dP = LdDu(dp + off + P.sI);
        const float2 rJp = Ld2(rp + off + P.sJ), rJm = Ld2(rp + off - P.sJ);
        const unsigned dJp = LdDu(dp + off + P.sJ), dJm = LdDu(dp + off - P.sJ);
        const float2 RP = red(rP, dP, i + 1);
        // the pairs one row over have the opposite colour order: (i, j+-1, k) has the parity of (i+-1, j, k)
        const float2 RJp = red(rJp, dJp, i + 1), RJm = red(rJm, dJm, i - 1);
        // the red value across the pair boundary: the previous pair's second cell or the next pair's first cell
        float left = __shfl_up_sync(0xffffffffu, RC.y, 1);
        float right = __shfl_down_sync(0xffffffffu, RC.x, 1);
        if (P.lane == 0)
        {
            const long long cl = P.base + off - 1;
            const int kl = P.k0 - 1; // may be -1: then the cell is the previous row's last, a ring cell (du 0)
            left = ((i + P.j + kl) & 1) == 0 ? r[cl] * inv[du[cl] & 0x7Fu] : 0.f;
        }
        if (P.lane == 31)
        {
            const long long cr = P.base + off + 2;
            right = ((i + P.j + P.k0 + 2) & 1) == 0 ? r[cr] * inv[du[cr] & 0x7Fu] : 0.f;
        }
        const bool firstRed = ((i + P.j + P.k0) & 1) == 0;
        float2 out;
        if (firstRed)
        {
            // black is the second cell: k neighbours are the first cell and the next pair's first
            const float s = ((RP.y + RM.y) + (RJp.y + RJm.y)) + (RC.x + right);
            out = make_float2(RC.x, (rC.y + g * s) * inv[(dC >> 8) & 0x7Fu]);
        }
        else
        {
            const float s = ((RP.x + RM.x) + (RJp.x + RJm.x)) + (left + RC.y);
            out = make_float2((rC.x + g * s) * inv[dC & 0x7Fu], RC.y);
        }
        if (P.valid) *reinterpret_cast<float2 *>(ep + off) = out;
        RM = RC;
        RC = RP;
        rC = rP;
        dC = dP;
    }
}

// One colour of a red-black sweep, in place: e_c = (r_c + gamma * sum of the six neighbours) / diag_c. Every value
// read has the other colour, so nothing read changes during the sweep. kDot (the last sweep of the level-0 V-cycle,
// whose result is the CG's z): also (sum r.z, sum z, sum r) into the scalar block of the iteration's parity.
template <bool kDot>
__global__ void __launch_bounds__(kPairThreads) k_pair_half(LevelView v, const uint8_t *__restrict__ du,
                                                            const float *__restrict__ r, float *e, int colour,
                                                            Reducer R, const int *it, int baseEven, int baseOdd)
{
    float facc[3] = {0.f, 0.f, 0.f}; // a thread's (at most 2 x kPairS) terms in FP32, the block and grid sums in FP64
    __shared__ float inv[32];
    FillInverse(inv, v.gamma);
    const PairPos P = PairStart(v);
    const float g = (float)v.gamma;
    const float *rp = r + P.base;
    const uint8_t *dp = du + P.base;
    float *ep = e + P.base;
    float2 eM = Ld2(ep - P.sI), eC = Ld2(ep);
    int off = 0;
    for (int i = P.i0; i < P.i1; i++, off += P.sI)
    {
        const float2 eP = Ld2(ep + off + P.sI);
        const float2 eJp = Ld2(ep + off + P.sJ), eJm = Ld2(ep + off - P.sJ);
        const float2 rc = Ld2(rp + off);
        const unsigned d = LdDu(dp + off);
        float left = __shfl_up_sync(0xffffffffu, eC.y, 1);
        float right = __shfl_down_sync(0xffffffffu, eC.x, 1);
        if (P.lane == 0) left = ep[off - 1];
        if (P.lane == 31) right = ep[off + 2];
        const bool second = ((i + P.j + P.k0) & 1) != colour; // the cell of this colour is the pair's second
        float s, rv;
        unsigned units;
        if (second)
        {
            s = ((eP.y + eM.y) + (eJp.y + eJm.y)) + (eC.x + right);
            rv = rc.y;
            units = (d >> 8) & 0x7Fu;
        }
        else
        {
            s = ((eP.x + eM.x) + (eJp.x + eJm.x)) + (left + eC.y);
            rv = rc.x;
            units = d & 0x7Fu;
        }
        const float nv = (rv + g * s) * inv[units];
        if (P.valid)
        {
            ep[off + (second ? 1 : 0)] = nv;
            if (kDot)
            {
                const float z0 = second ? eC.x : nv, z1 = second ? nv : eC.y;
                facc[0] += rc.x * z0 + rc.y * z1;
                facc[1] += z0 + z1;
                facc[2] += rc.x + rc.y;
            }
        }
        eM = eC;
        eC = eP;
    }
    if (kDot)
    {
        double acc[3] = {facc[0], facc[1], facc[2]};
        GridReduce<3>(R, acc, (*it & 1) ? baseOdd : baseEven);
    }
}

// res = r - M e
__global__ void __launch_bounds__(kPairThreads) k_pair_residual(LevelView v, const uint8_t *__restrict__ du,
                                                                const float *__restrict__ r,
                                                                const float *__restrict__ e, float *__restrict__ res)
{
    const PairPos P = PairStart(v);
    const float g = (float)v.gamma, hg = 0.5f * (float)v.gamma;
    const float *ep = e + P.base;
    const float *rp = r + P.base;
    const uint8_t *dp = du + P.base;
    float *op = res + P.base;
    float2 eM = Ld2(ep - P.sI), eC = Ld2(ep);
    int off = 0;
    for (int i = P.i0; i < P.i1; i++, off += P.sI)
    {
        const float2 eP = Ld2(ep + off + P.sI);
        const float2 eJp = Ld2(ep + off + P.sJ), eJm = Ld2(ep + off - P.sJ);
        const float2 rc = Ld2(rp + off);
        const unsigned d = LdDu(dp + off);
        float left = __shfl_up_sync(0xffffffffu, eC.y, 1);
        float right = __shfl_down_sync(0xffffffffu, eC.x, 1);
        if (P.lane == 0) left = ep[off - 1];
        if (P.lane == 31) right = ep[off + 2];
        if (P.valid && (d & 0x8080u))
        {
            const float s0 = ((eP.x + eM.x) + (eJp.x + eJm.x)) + (left + eC.y);
            const float s1 = ((eP.y + eM.y) + (eJp.y + eJm.y)) + (eC.x + right);
            float2 o;
            o.x = (d & 0x80u) ? rc.x - (hg * (float)(d & 0x7Fu) * eC.x - g * s0) : 0.f;
            o.y = (d & 0x8000u) ? rc.y - (hg * (float)((d >> 8) & 0x7Fu) * eC.y - g * s1) : 0.f;
            *reinterpret_cast<float2 *>(op + off) = o;
        }
        eM = eC;
        eC = eP;
    }
}

// ---------------------------------------------------------------------------------------------------------------
// the same on a stretched level: the six coefficients of a cell come from the level's FP32 width and gap tables and
// the diagonal from its code byte (CodeStencil, nb_device.cuh); the neighbour sum stays unmasked (vectors are zero
// off the unknowns), weighted per direction. The first sweep from zero is a red pass writing r/diag (and zero on
// black) followed by a black pass.
// ---------------------------------------------------------------------------------------------------------------
// The table entries of a pair's two cells (i, j, k0 + h) that do not change along a thread's march over the planes
// i: Width x of row j and 1/FaceGap x on its sides, Width z of both cells and 1/FaceGap z on their sides. With them
// a plane costs two table reads (Width y and the upper 1/FaceGap y; the lower one is the plane before's upper) where
// LevelCoefs reads nine; the products are LevelCoefs' own, in its order.
struct StPair
{
    float wx, igx0, igx1;
    float wz[2], igz[3];
};

__device__ __forceinline__ StPair StPairOf(const LevelView &v, int j, int k0)
{
    StPair S;
    S.wx = v.w32[0][j + 1];
    S.igx0 = v.ig32[0][j];
    S.igx1 = v.ig32[0][j + 1];
    S.wz[0] = v.w32[2][k0 + 1];
    S.wz[1] = v.w32[2][k0 + 2];
    S.igz[0] = v.ig32[2][k0];
    S.igz[1] = v.ig32[2][k0 + 1];
    S.igz[2] = v.ig32[2][k0 + 2];
    return S;
}

// LevelCoefs of cell (i, j, k0 + h) from the pair's entries and plane i's Width y and 1/FaceGap y below and above
__device__ __forceinline__ void StCoefs(const StPair &S, int h, float wy, float igyLo, float igyHi, float c[6])
{
    const float wz = S.wz[h];
    const float ax = wy * wz, ay = S.wx * wz, az = S.wx * wy;
    c[0] = ay * igyHi;
    c[1] = ay * igyLo;
    c[2] = ax * S.igx1;
    c[3] = ax * S.igx0;
    c[4] = az * S.igz[h + 1];
    c[5] = az * S.igz[h];
}

// CodeStencil's diagonal from given coefficients: the FLUID neighbours' coefficients, then the Dirichlet ones (a
// ring neighbour's weighted by the ring factor)
__device__ __forceinline__ float StDiag(const LevelView &v, int i, int j, int k, long long c, unsigned code,
                                        const float cq[6])
{
    const unsigned m = code & CODE_FLUID_MASK;
    float d = 0.f;
#pragma unroll
    for (int q = 0; q < 6; q++)
        if (m >> q & 1u) d += cq[q];
    if (code & CODE_DIRICHLET)
        for (int q = 0; q < 6; q++)
        {
            const int t = v.types[c + NbrOffset(v, q)];
            if (IsDirichlet(t))
            {
                const int ni = i + (q == 0) - (q == 1), nj = j + (q == 2) - (q == 3), nk = k + (q == 4) - (q == 5);
                d += OnRing(v, ni, nj, nk) ? cq[q] * LevelRingFactor<float>(v, i, j, k, q) : cq[q];
            }
        }
    return d;
}

// sum_q c_q x_q over the six neighbours of unknown cell (i, j, k0 + h) and its diagonal; neighbours in NbrOffset order
__device__ __forceinline__ float StSum(const LevelView &v, const StPair &S, int h, float wy, float igyLo, float igyHi,
                                       int i, int j, int k, long long c, unsigned code, float nP, float nM, float nJp,
                                       float nJm, float nKp, float nKm, float &diag)
{
    float cq[6];
    StCoefs(S, h, wy, igyLo, igyHi, cq);
    diag = StDiag(v, i, j, k, c, code, cq);
    return ((cq[0] * nP + cq[1] * nM) + (cq[2] * nJp + cq[3] * nJm)) + (cq[4] * nKp + cq[5] * nKm);
}

template <bool kDot, bool kFirst>
__global__ void __launch_bounds__(kPairThreads) k_pair_half_st(LevelView v, const float *__restrict__ r, float *e,
                                                               int colour, Reducer R, const int *it, int baseEven,
                                                               int baseOdd)
{
    float facc[3] = {0.f, 0.f, 0.f};
    const PairPos P = PairStart(v);
    const float *rp = r + P.base;
    const uint8_t *cp = v.code + P.base;
    float *ep = e + P.base;
    float2 eM = kFirst ? make_float2(0.f, 0.f) : Ld2(ep - P.sI), eC = kFirst ? make_float2(0.f, 0.f) : Ld2(ep);
    const StPair SP = StPairOf(v, P.j, P.k0);
    float igyLo = v.ig32[1][P.i0];
    int off = 0;
    for (int i = P.i0; i < P.i1; i++, off += P.sI)
    {
        const float wy = v.w32[1][i + 1], igyHi = v.ig32[1][i + 1];
        float2 eP = make_float2(0.f, 0.f), eJp = eP, eJm = eP;
        if (!kFirst)
        {
            eP = Ld2(ep + off + P.sI);
            eJp = Ld2(ep + off + P.sJ);
            eJm = Ld2(ep + off - P.sJ);
        }
        const float2 rc = Ld2(rp + off);
        const unsigned d = LdDu(cp + off);
        float left = 0.f, right = 0.f;
        if (!kFirst)
        {
            left = __shfl_up_sync(0xffffffffu, eC.y, 1);
            right = __shfl_down_sync(0xffffffffu, eC.x, 1);
            if (P.lane == 0) left = ep[off - 1];
            if (P.lane == 31) right = ep[off + 2];
        }
        const bool second = ((i + P.j + P.k0) & 1) != colour; // the cell of this colour is the pair's second
        const int h = second ? 1 : 0, k = P.k0 + h;
        const unsigned code = (d >> (8 * h)) & 0xFFu;
        float nv = 0.f;
        if (code & CODE_UNKNOWN)
        {
            float diag, s = 0.f;
            const long long c = P.base + off + h;
            if (kFirst)
            {
                float cq[6];
                StCoefs(SP, h, wy, igyLo, igyHi, cq);
                diag = StDiag(v, i, P.j, k, c, code, cq);
            }
            else if (second)
                s = StSum(v, SP, h, wy, igyLo, igyHi, i, P.j, k, c, code, eP.y, eM.y, eJp.y, eJm.y, right, eC.x, diag);
            else
                s = StSum(v, SP, h, wy, igyLo, igyHi, i, P.j, k, c, code, eP.x, eM.x, eJp.x, eJm.x, eC.y, left, diag);
            nv = diag != 0.f ? ((second ? rc.y : rc.x) + s) / diag : 0.f;
        }
        if (P.valid)
        {
            if (kFirst) // red from zero: the black cells start at zero
                *reinterpret_cast<float2 *>(ep + off) = second ? make_float2(0.f, nv) : make_float2(nv, 0.f);
            else
                ep[off + h] = nv;
            if (kDot)
            {
                const float z0 = second ? eC.x : nv, z1 = second ? nv : eC.y;
                facc[0] += rc.x * z0 + rc.y * z1;
                facc[1] += z0 + z1;
                facc[2] += rc.x + rc.y;
            }
        }
        eM = eC;
        eC = eP;
        igyLo = igyHi;
    }
    if (kDot)
    {
        double acc[3] = {facc[0], facc[1], facc[2]};
        GridReduce<3>(R, acc, (*it & 1) ? baseOdd : baseEven);
    }
}

__global__ void __launch_bounds__(kPairThreads) k_pair_residual_st(LevelView v, const float *__restrict__ r,
                                                                   const float *__restrict__ e,
                                                                   float *__restrict__ res)
{
    const PairPos P = PairStart(v);
    const float *ep = e + P.base;
    const float *rp = r + P.base;
    const uint8_t *cp = v.code + P.base;
    float *op = res + P.base;
    float2 eM = Ld2(ep - P.sI), eC = Ld2(ep);
    const StPair SP = StPairOf(v, P.j, P.k0);
    float igyLo = v.ig32[1][P.i0];
    int off = 0;
    for (int i = P.i0; i < P.i1; i++, off += P.sI)
    {
        const float wy = v.w32[1][i + 1], igyHi = v.ig32[1][i + 1];
        const float2 eP = Ld2(ep + off + P.sI);
        const float2 eJp = Ld2(ep + off + P.sJ), eJm = Ld2(ep + off - P.sJ);
        const float2 rc = Ld2(rp + off);
        const unsigned d = LdDu(cp + off);
        float left = __shfl_up_sync(0xffffffffu, eC.y, 1);
        float right = __shfl_down_sync(0xffffffffu, eC.x, 1);
        if (P.lane == 0) left = ep[off - 1];
        if (P.lane == 31) right = ep[off + 2];
        if (P.valid && (d & 0x8080u))
        {
            float2 o = make_float2(0.f, 0.f);
            const long long c = P.base + off;
            float diag;
            if (d & 0x80u)
            {
                const float s = StSum(v, SP, 0, wy, igyLo, igyHi, i, P.j, P.k0, c, d & 0xFFu, eP.x, eM.x, eJp.x,
                                      eJm.x, eC.y, left, diag);
                o.x = rc.x - (diag * eC.x - s);
            }
            if (d & 0x8000u)
            {
                const float s = StSum(v, SP, 1, wy, igyLo, igyHi, i, P.j, P.k0 + 1, c + 1, (d >> 8) & 0xFFu, eP.y,
                                      eM.y, eJp.y, eJm.y, right, eC.x, diag);
                o.y = rc.y - (diag * eC.y - s);
            }
            *reinterpret_cast<float2 *>(op + off) = o;
        }
        eM = eC;
        eC = eP;
        igyLo = igyHi;
    }
}

void LaunchPairHalfSt(const LevelView &v, const float *r, float *e, int colour, bool first, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    if (first)
        k_pair_half_st<false, true><<<PairGrid(v), kPairThreads, 0, st>>>(v, r, e, colour, Reducer{}, nullptr, 0, 0);
    else
        k_pair_half_st<false, false><<<PairGrid(v), kPairThreads, 0, st>>>(v, r, e, colour, Reducer{}, nullptr, 0, 0);
}

void LaunchPairHalfStDot(const LevelView &v, const float *r, float *e, int colour, const Reducer &R, const int *it,
                         int baseEven, int baseOdd, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_pair_half_st<true, false><<<PairGrid(v, kReduceS), kPairThreads, 0, st>>>(v, r, e, colour, R, it, baseEven,
                                                                               baseOdd);
}

void LaunchPairResidualSt(const LevelView &v, const float *r, const float *e, float *res, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_pair_residual_st<<<PairGrid(v), kPairThreads, 0, st>>>(v, r, e, res);
}

void LaunchPairFirst(const LevelView &v, const uint8_t *du, const float *r, float *e, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_pair_first<<<PairGrid(v), kPairThreads, 0, st>>>(v, du, r, e);
}

void LaunchPairHalf(const LevelView &v, const uint8_t *du, const float *r, float *e, int colour, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_pair_half<false><<<PairGrid(v), kPairThreads, 0, st>>>(v, du, r, e, colour, Reducer{}, nullptr, 0, 0);
}

void LaunchPairHalfDot(const LevelView &v, const uint8_t *du, const float *r, float *e, int colour, const Reducer &R,
                       const int *it, int baseEven, int baseOdd, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_pair_half<true><<<PairGrid(v, kReduceS), kPairThreads, 0, st>>>(v, du, r, e, colour, R, it, baseEven, baseOdd);
}

void LaunchPairResidual(const LevelView &v, const uint8_t *du, const float *r, const float *e, float *res,
                        cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_pair_residual<<<PairGrid(v), kPairThreads, 0, st>>>(v, du, r, e, res);
}

// ---------------------------------------------------------------------------------------------------------------
// transfers between a pair level and the next coarser level (the operators of k_prolong / k_restrict)
// ---------------------------------------------------------------------------------------------------------------
// Per fine cell: 0x80 for an unknown, plus in the low six bits the weight (in 1/64) that the Neumann-aware
// prolongation moves from the cell's SOLID coarse contributors onto its parent. Coarse vectors are zero at SOLID
// cells, so P e_c at a fine unknown = the plain trilinear sum + extra/64 * e_c[parent], and R = P^T.
// A colour-split fine level keeps the red cells' bytes only (its transfers run over the red cells).
__global__ void k_build_pext(LevelView fv, LevelView cv, uint8_t *pext)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < fv.cells;
         c += (long long)gridDim.x * blockDim.x)
    {
        const int d = (int)(c % fv.Nz);
        const long long rr = c / fv.Nz;
        const int b = (int)(rr % fv.Nx), a = (int)(rr / fv.Nx);
        if (fv.sRS && ((a + b + d) & 1)) continue;
        const long long o = VecIdx(fv, a, b, d);
        const bool interior = a > 0 && a < fv.Ny - 1 && b > 0 && b < fv.Nx - 1 && d > 0 && d < fv.Nz - 1;
        if (!interior || fv.types[c] != FLUID) { pext[o] = 0; continue; }
        const int A = (a + 1) >> 1, D = (d + 1) >> 1;
        const int si = (a & 1) ? -1 : 1, sk = (d & 1) ? -1 : 1;
        // along x (j): the parent and the neighbour on the cell's side, 3/4 and 1/4; with x groups (xp) a parent of
        // one child takes all of it
        int B = (b + 1) >> 1, B2 = B + ((b & 1) ? -1 : 1), wj0 = 3, wj1 = 1;
        if (fv.xp)
        {
            const int x = fv.xp[b];
            B = XpParent(x);
            B2 = XpOther(x);
            if (XpSingle(x)) { wj0 = 4; wj1 = 0; }
        }
        const int w[2] = {3, 1}, wj[2] = {wj0, wj1};
        unsigned extra = 0;
        for (int di = 0; di < 2; di++)
            for (int dj = 0; dj < 2; dj++)
                for (int dk = 0; dk < 2; dk++)
                {
                    if (!(di | dj | dk)) continue;
                    const long long cc = (long long)(A + di * si) * cv.sI + (long long)(dj ? B2 : B) * cv.sJ +
                                         (D + dk * sk);
                    if (cv.types[cc] == SOLID) extra += (unsigned)(w[di] * wj[dj] * w[dk]);
                }
        pext[o] = (uint8_t)(0x80u | extra);
    }
}

void LaunchBuildPext(const LevelView &fine, const LevelView &coarse, uint8_t *pext, cudaStream_t st)
{
    int blocks = (int)((fine.cells + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    NB_COUNT_LAUNCH();
    k_build_pext<<<blocks, 256, 0, st>>>(fine, coarse, pext);
}

// e_f += P e_c on the fine unknowns; one thread per fine pair (k0 even: parents k0/2 and k0/2 + 1 along k).
// kX: the coarsening keeps some x cells whole (LevelView::xp gives the x parent, the other contributor, their weights)
template <bool kX>
__global__ void __launch_bounds__(kPairThreads) k_pair_prolong(LevelView fv, LevelView cv,
                                                               const uint8_t *__restrict__ pext,
                                                               const float *__restrict__ ec, float *ef)
{
    const PairPos P = PairStart(fv);
    const int m = P.k0 >> 1;
    int off = 0;
    for (int a = P.i0; a < P.i1; a++, off += P.sI)
    {
        const unsigned x = LdDu(pext + P.base + off);
        if (!P.valid || !(x & 0x8080u)) continue;
        const int b = P.j;
        const int A = (a + 1) >> 1, A2 = A + ((a & 1) ? -1 : 1);
        int B = (b + 1) >> 1, B2 = B + ((b & 1) ? -1 : 1);
        bool one = false;
        if constexpr (kX)
        {
            const int xq = fv.xp[b];
            B = XpParent(xq);
            B2 = XpOther(xq);
            one = XpSingle(xq);
        }
        const float *r00 = ec + (long long)A * cv.sI + (long long)B * cv.sJ + m;
        const float *r01 = ec + (long long)A * cv.sI + (long long)B2 * cv.sJ + m;
        const float *r10 = ec + (long long)A2 * cv.sI + (long long)B * cv.sJ + m;
        const float *r11 = ec + (long long)A2 * cv.sI + (long long)B2 * cv.sJ + m;
        // rows weighted 3/4 (parent's row and plane) and 1/4 across i and j, then along k
        float lo, hi;
        if (!kX)
        {
            lo = 0.5625f * r00[0] + 0.1875f * (r01[0] + r10[0]) + 0.0625f * r11[0];
            hi = 0.5625f * r00[1] + 0.1875f * (r01[1] + r10[1]) + 0.0625f * r11[1];
        }
        else if (one) // one x child: the parent's row and column only along x
        {
            lo = 0.75f * r00[0] + 0.25f * r10[0];
            hi = 0.75f * r00[1] + 0.25f * r10[1];
        }
        else
        {
            lo = 0.75f * (0.75f * r00[0] + 0.25f * r01[0]) + 0.25f * (0.75f * r10[0] + 0.25f * r11[0]);
            hi = 0.75f * (0.75f * r00[1] + 0.25f * r01[1]) + 0.25f * (0.75f * r10[1] + 0.25f * r11[1]);
        }
        float2 v = *reinterpret_cast<float2 *>(ef + P.base + off);
        if (x & 0x80u) v.x += (0.75f * lo + 0.25f * hi) + (float)(x & 0x3Fu) * (1.0f / 64.0f) * r00[0];
        if (x & 0x8000u) v.y += (0.75f * hi + 0.25f * lo) + (float)((x >> 8) & 0x3Fu) * (1.0f / 64.0f) * r00[1];
        *reinterpret_cast<float2 *>(ef + P.base + off) = v;
    }
}

void LaunchPairProlong(const LevelView &fine, const LevelView &coarse, const uint8_t *pext, const float *eCoarse,
                       float *eFine, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    if (fine.xp) k_pair_prolong<true><<<PairGrid(fine), kPairThreads, 0, st>>>(fine, coarse, pext, eCoarse, eFine);
    else k_pair_prolong<false><<<PairGrid(fine), kPairThreads, 0, st>>>(fine, coarse, pext, eCoarse, eFine);
}

// r_c = R res_f = P^T res_f at the coarse unknowns. A thread owns one coarse cell (K along the 32 lanes, J across
// the 8 warps) and marches along I: fine planes 2I-2 .. 2I+1 enter as their (j, k)-weighted 4x4 sums T(a), each
// fine plane summed once and kept for the next coarse plane; the children's moved weights enter as X(a).

__device__ __forceinline__ void RestrictPlane(const LevelView &fv, const uint8_t *pext, const float *res, int a,
                                              int J, int K, float &T, float &X)
{
    T = 0.f;
    X = 0.f;
    if (a > fv.Ny - 1) return;
    const float wt[4] = {0.25f, 0.75f, 0.75f, 0.25f};
#pragma unroll
    for (int dj = 0; dj < 4; dj++)
    {
        const int b = 2 * J - 2 + dj;
        if (b > fv.Nx - 1) continue;
        const long long row = (long long)a * fv.sI + (long long)b * fv.sJ + 2 * K - 2;
        const float2 u = *reinterpret_cast<const float2 *>(res + row);
        const float2 w = *reinterpret_cast<const float2 *>(res + row + 2);
        T += wt[dj] * ((0.25f * u.x + 0.75f * u.y) + (0.75f * w.x + 0.25f * w.y));
        if (dj == 1 || dj == 2)
        {
            // children 2K-1 (u.y) and 2K (w.x) of this row
            X += (float)(pext[row + 1] & 0x3Fu) * u.y + (float)(pext[row + 2] & 0x3Fu) * w.x;
        }
    }
    X *= 1.0f / 64.0f;
}

// The same plane sum where the coarsening keeps some x cells whole: the x taps of coarse J (XrTaps) replace the
// fixed 2J-2 .. 2J+1; a warp holds one J, so the skipped taps do not diverge.
__device__ __forceinline__ void RestrictPlaneX(const LevelView &fv, const uint8_t *pext, const float *res, int a,
                                               int K, const int (&bq)[4], const float (&wq)[4], bool two, float &T,
                                               float &X)
{
    T = 0.f;
    X = 0.f;
    if (a > fv.Ny - 1) return;
#pragma unroll
    for (int dj = 0; dj < 4; dj++)
    {
        if (wq[dj] == 0.f) continue;
        const long long row = (long long)a * fv.sI + (long long)bq[dj] * fv.sJ + 2 * K - 2;
        const float2 u = *reinterpret_cast<const float2 *>(res + row);
        const float2 w = *reinterpret_cast<const float2 *>(res + row + 2);
        T += wq[dj] * ((0.25f * u.x + 0.75f * u.y) + (0.75f * w.x + 0.25f * w.y));
        if (dj == 1 || (dj == 2 && two))
            X += (float)(pext[row + 1] & 0x3Fu) * u.y + (float)(pext[row + 2] & 0x3Fu) * w.x;
    }
    X *= 1.0f / 64.0f;
}

template <bool kX>
__global__ void __launch_bounds__(256) k_pair_restrict(LevelView fv, LevelView cv, const uint8_t *__restrict__ pext,
                                                       const float *__restrict__ res, float *__restrict__ rc)
{
    const int K = 1 + blockIdx.x * 32 + threadIdx.x, J = 1 + blockIdx.y * 8 + threadIdx.y;
    if (K > cv.Nz - 2 || J > cv.Nx - 2) return;
    // coarse planes in chunks of S (grid.z as the host sized it, MarchPlanes)
    const int S = (cv.Ny - 2 + (int)gridDim.z - 1) / (int)gridDim.z;
    const int I0 = 1 + (int)blockIdx.z * S, I1 = min(I0 + S, cv.Ny - 1);
    if (I0 >= I1) return;
    int bq[4] = {0, 0, 0, 0};
    float wq[4] = {0.f, 0.f, 0.f, 0.f};
    bool two = false;
    if constexpr (kX) XrTaps<float>(fv.xr[J], bq, wq, two);
    auto plane = [&](int a, float &T, float &X) {
        if constexpr (kX) RestrictPlaneX(fv, pext, res, a, K, bq, wq, two, T, X);
        else RestrictPlane(fv, pext, res, a, J, K, T, X);
    };
    float Tm2, Tm1, Xm1, Xdummy;
    plane(2 * I0 - 2, Tm2, Xdummy);
    plane(2 * I0 - 1, Tm1, Xm1);
    for (int I = I0; I < I1; I++)
    {
        float T0, X0, T1, X1;
        plane(2 * I, T0, X0);
        plane(2 * I + 1, T1, X1);
        const long long c = (long long)I * cv.sI + (long long)J * cv.sJ + K;
        if (cv.code[c] & CODE_UNKNOWN)
            rc[c] = ((0.25f * Tm2 + 0.75f * Tm1) + (0.75f * T0 + 0.25f * T1)) + (Xm1 + X0);
        Tm2 = T0;
        Tm1 = T1;
        Xm1 = X1;
    }
}

void LaunchPairRestrict(const LevelView &fine, const LevelView &coarse, const uint8_t *pext, const float *resFine,
                        float *rCoarse, cudaStream_t st)
{
    const long long perPlane = (long long)((coarse.Nz - 2 + 31) / 32) * ((coarse.Nx - 2 + 7) / 8);
    const int S = MarchPlanes(coarse.Ny - 2, perPlane);
    const dim3 grid((unsigned)((coarse.Nz - 2 + 31) / 32), (unsigned)((coarse.Nx - 2 + 7) / 8),
                    (unsigned)((coarse.Ny - 2 + S - 1) / S));
    NB_COUNT_LAUNCH();
    if (fine.xr) k_pair_restrict<true><<<grid, dim3(32, 8), 0, st>>>(fine, coarse, pext, resFine, rCoarse);
    else k_pair_restrict<false><<<grid, dim3(32, 8), 0, st>>>(fine, coarse, pext, resFine, rCoarse);
}

// ---------------------------------------------------------------------------------------------------------------
// PCG on level 0 (the semantics of k_update_p_apply / k_dot / k_update_xr in nb_kernels.cu)
// ---------------------------------------------------------------------------------------------------------------
// n (the unknowns) comes from S[slotN] on the device (a captured iteration outlives a same-shape layout change)
__device__ __forceinline__ double RzEffP(const double *S, int base, double n, int singular)
{
    return singular ? S[base] - (S[base + 1] / n) * S[base + 2] : S[base];
}

// p_new = U (z - mean + beta p_old), q = M p_new, sum p_new.q; U = 1 on unknowns (needed only when the mean of z is
// removed: elsewhere z and p_old are zero already).
// kSt: a stretched level, `du` is then the level's code array (its unknown flag is the same bit)
template <bool kSingular, bool kSt>
__global__ void __launch_bounds__(kPairThreads)
    k_pair_papply(LevelView v, const uint8_t *__restrict__ du, const float *__restrict__ z, float *p0, float *p1,
                  float *__restrict__ q, Reducer R, const double *S, const int *it, int baseEven, int baseOdd, int slotN,
                  int slotPQ)
{
    const int iter = *it, par = iter & 1;
    const float *__restrict__ pIn = par ? p1 : p0;
    float *__restrict__ pOut = par ? p0 : p1;
    const int baseNew = par ? baseOdd : baseEven, baseOld = par ? baseEven : baseOdd;
    const double n = S[slotN];
    const double beta = iter == 0 ? 0.0 : RzEffP(S, baseNew, n, kSingular) / RzEffP(S, baseOld, n, kSingular);
    const float b = (float)beta;
    const float mean = kSingular ? (float)(S[baseNew + 1] / n) : 0.f;
    const PairPos P = PairStart(v);
    const float g = (float)v.gamma, hg = 0.5f * (float)v.gamma;
    const float *zp = z + P.base;
    const float *pp = pIn + P.base;
    const uint8_t *dp = du + P.base;
    auto pnew = [&](int o) {
        const float2 zz = Ld2(zp + o), pv = Ld2(pp + o);
        float2 out = make_float2((zz.x - mean) + b * pv.x, (zz.y - mean) + b * pv.y);
        if (kSingular)
        {
            const unsigned d = LdDu(dp + o);
            out.x *= Unk(d);
            out.y *= Unk(d >> 8);
        }
        return out;
    };
    auto pnew1 = [&](long long c) {
        float x = (z[c] - mean) + b * pIn[c];
        if (kSingular) x *= Unk(du[c]);
        return x;
    };
    float2 NM = pnew(-P.sI), NC = pnew(0);
    float facc = 0.f;
    StPair SP{};
    float igyLo = 0.f;
    if (kSt)
    {
        SP = StPairOf(v, P.j, P.k0);
        igyLo = v.ig32[1][P.i0];
    }
    int off = 0;
    for (int i = P.i0; i < P.i1; i++, off += P.sI)
    {
        const float wy = kSt ? v.w32[1][i + 1] : 0.f, igyHi = kSt ? v.ig32[1][i + 1] : 0.f;
        const float2 NP = pnew(off + P.sI);
        const float2 NJp = pnew(off + P.sJ), NJm = pnew(off - P.sJ);
        const unsigned d = LdDu(dp + off);
        float left = __shfl_up_sync(0xffffffffu, NC.y, 1);
        float right = __shfl_down_sync(0xffffffffu, NC.x, 1);
        if (P.lane == 0) left = pnew1(P.base + off - 1);
        if (P.lane == 31) right = pnew1(P.base + off + 2);
        const float s0 = ((NP.x + NM.x) + (NJp.x + NJm.x)) + (left + NC.y);
        const float s1 = ((NP.y + NM.y) + (NJp.y + NJm.y)) + (NC.x + right);
        float2 qq;
        if (kSt)
        {
            qq = make_float2(0.f, 0.f);
            float diag;
            if (d & 0x80u)
            {
                const float s = StSum(v, SP, 0, wy, igyLo, igyHi, i, P.j, P.k0, P.base + off, d & 0xFFu, NP.x, NM.x,
                                      NJp.x, NJm.x, NC.y, left, diag);
                qq.x = diag * NC.x - s;
            }
            if (d & 0x8000u)
            {
                const float s = StSum(v, SP, 1, wy, igyLo, igyHi, i, P.j, P.k0 + 1, P.base + off + 1, (d >> 8) & 0xFFu,
                                      NP.y, NM.y, NJp.y, NJm.y, right, NC.x, diag);
                qq.y = diag * NC.y - s;
            }
        }
        else
        {
            qq.x = Unk(d) * (hg * (float)(d & 0x7Fu) * NC.x - g * s0);
            qq.y = Unk(d >> 8) * (hg * (float)((d >> 8) & 0x7Fu) * NC.y - g * s1);
        }
        if (P.valid)
        {
            *reinterpret_cast<float2 *>(pOut + P.base + off) = NC;
            *reinterpret_cast<float2 *>(q + P.base + off) = qq;
            facc += NC.x * qq.x + NC.y * qq.y;
        }
        NM = NC;
        NC = NP;
        igyLo = igyHi;
    }
    double acc[1] = {facc};
    GridReduce<1>(R, acc, slotPQ);
}

void LaunchPairPApply(const LevelView &v, const uint8_t *du, const float *z, float *p0, float *p1, float *q,
                      const Reducer &R, const double *S, const int *it, int baseEven, int baseOdd, int slotN,
                      int singular, int slotPQ, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    const dim3 grid = PairGrid(v, kReduceS);
    const uint8_t *bytes = v.stretched ? v.code : du;
#define NB_PAPPLY(SING, ST)                                                                                        \
    k_pair_papply<SING, ST><<<grid, kPairThreads, 0, st>>>(v, bytes, z, p0, p1, q, R, S, it, baseEven, baseOdd, slotN, \
                                                           slotPQ)
    if (singular)
    {
        if (v.stretched) NB_PAPPLY(true, true);
        else NB_PAPPLY(true, false);
    }
    else
    {
        if (v.stretched) NB_PAPPLY(false, true);
        else NB_PAPPLY(false, false);
    }
#undef NB_PAPPLY
}

// ---------------------------------------------------------------------------------------------------------------
// FP64 refinement step on level 0 (the semantics of k_residual64<float, true> in nb_exact.cu for a uniform 3D grid)
// ---------------------------------------------------------------------------------------------------------------
// x_out = x_in + e; r = sfac (b - A x_out) in FP32; (sum (b - A x_out)^2, sum (b - A x_out)) in FP64. A is the
// reference's matrix on a uniform grid: scale (sum of the FLUID neighbours - diag units / 2 x), c_q = 1 and scale =
// 1/dh^2 (FaceCoefs3D, MatrixScale3D, PressureSolver3D.cpp:34-63). x_in and e are zero off the unknowns, so the
// neighbour sum runs over all six; the sum's order differs from the per-cell kernel's, within FP64 rounding.
__device__ __forceinline__ double2 Ld2d(const double *p) { return *reinterpret_cast<const double2 *>(p); }

// swap (may be null): when *swap is odd, x_in and x_out trade places
__global__ void __launch_bounds__(kPairThreads)
    k_pair_refine64(LevelView v, const uint8_t *__restrict__ du, const double *__restrict__ b,
                    const double *xin0, const float *__restrict__ e, double *xout0,
                    float *__restrict__ r, double scale, double sfac, Reducer R, int slot, const int *swap)
{
    const bool sw = swap && (*swap & 1);
    const double *__restrict__ xin = sw ? xout0 : xin0;
    double *__restrict__ xout = sw ? const_cast<double *>(xin0) : xout0;
    const PairPos P = PairStart(v);
    auto X = [&](int o) {
        const double2 a = Ld2d(xin + P.base + o);
        const float2 f = Ld2(e + P.base + o);
        return make_double2(a.x + (double)f.x, a.y + (double)f.y);
    };
    auto X1 = [&](long long c) { return xin[c] + (double)e[c]; };
    double2 XM = X(-P.sI), XC = X(0);
    double acc[2] = {0.0, 0.0};
    int off = 0;
    for (int i = P.i0; i < P.i1; i++, off += P.sI)
    {
        const double2 XP = X(off + P.sI), XJp = X(off + P.sJ), XJm = X(off - P.sJ);
        const double2 bb = Ld2d(b + P.base + off);
        const unsigned d = LdDu(du + P.base + off);
        double left = __shfl_up_sync(0xffffffffu, XC.y, 1);
        double right = __shfl_down_sync(0xffffffffu, XC.x, 1);
        if (P.lane == 0) left = X1(P.base + off - 1);
        if (P.lane == 31) right = X1(P.base + off + 2);
        const double s0 = ((XP.x + XM.x) + (XJp.x + XJm.x)) + (left + XC.y);
        const double s1 = ((XP.y + XM.y) + (XJp.y + XJm.y)) + (XC.x + right);
        const double r0 = (d & 0x80u) ? bb.x - scale * (s0 - 0.5 * (double)(d & 0x7Fu) * XC.x) : 0.0;
        const double r1 = (d & 0x8000u) ? bb.y - scale * (s1 - 0.5 * (double)((d >> 8) & 0x7Fu) * XC.y) : 0.0;
        if (P.valid)
        {
            *reinterpret_cast<double2 *>(xout + P.base + off) = XC;
            *reinterpret_cast<float2 *>(r + P.base + off) = make_float2((float)(r0 * sfac), (float)(r1 * sfac));
            acc[0] += r0 * r0 + r1 * r1;
            acc[1] += r0 + r1;
        }
        XM = XC;
        XC = XP;
    }
    GridReduce<2>(R, acc, slot);
}

void LaunchPairRefine64(const LevelView &v, const uint8_t *du, const double *b, const double *xin, const float *e,
                        double *xout, float *r, double scale, double sfac, const Reducer &R, int slot,
                        cudaStream_t st, const int *swap)
{
    NB_COUNT_LAUNCH();
    k_pair_refine64<<<PairGrid(v, kReduceS), kPairThreads, 0, st>>>(v, du, b, xin, e, xout, r, scale, sfac, R,
                                                                      slot, swap);
}

// Whole-array kernels (every entry off the unknowns is zero): 16-byte loads over the level's cells.
constexpr int kLinBlocks = 148 * 8;

// (sum r.z, sum z, sum r)
__global__ void __launch_bounds__(256) k_lin_dot(long long cells, const float *__restrict__ r,
                                                 const float *__restrict__ z, Reducer R, const int *it, int baseEven,
                                                 int baseOdd)
{
    const int base = (*it & 1) ? baseOdd : baseEven;
    double acc[3] = {0.0, 0.0, 0.0};
    const long long n4 = cells >> 2, stride = (long long)gridDim.x * blockDim.x;
    const float4 *r4 = reinterpret_cast<const float4 *>(r), *z4 = reinterpret_cast<const float4 *>(z);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n4; t += stride)
    {
        const float4 a = r4[t], c = z4[t];
        acc[0] += (double)a.x * c.x + (double)a.y * c.y + (double)a.z * c.z + (double)a.w * c.w;
        acc[1] += ((double)c.x + c.y) + ((double)c.z + c.w);
        acc[2] += ((double)a.x + a.y) + ((double)a.z + a.w);
    }
    for (long long t = 4 * n4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cells; t += stride)
    {
        acc[0] += (double)r[t] * z[t];
        acc[1] += z[t];
        acc[2] += r[t];
    }
    GridReduce<3>(R, acc, base);
}

// alpha = rz / pq; x += alpha p; r -= alpha q; sum r.r; the last block advances the iteration counter
// bx of gx: this block among the launch's blocks (a grid-stride loop)
__device__ __forceinline__ void LinXR(long long cells, float *__restrict__ x, float *__restrict__ r, const float *p0,
                                      const float *p1, const float *__restrict__ q, const Reducer &R, const double *S,
                                      int *it, int baseEven, int baseOdd, int slotN, int singular, int slotPQ,
                                      int slotRR, int bx, int gx)
{
    const int par = *it & 1;
    const float *__restrict__ p = par ? p0 : p1;
    const int base = par ? baseOdd : baseEven;
    const float a = (float)(RzEffP(S, base, S[slotN], singular) / S[slotPQ]);
    double acc[1] = {0.0};
    const long long n4 = cells >> 2, stride = (long long)gx * blockDim.x;
    float4 *x4 = reinterpret_cast<float4 *>(x), *r4 = reinterpret_cast<float4 *>(r);
    const float4 *p4 = reinterpret_cast<const float4 *>(p), *q4 = reinterpret_cast<const float4 *>(q);
    for (long long t = bx * (long long)blockDim.x + threadIdx.x; t < n4; t += stride)
    {
        const float4 pv = p4[t], qv = q4[t];
        float4 xv = x4[t], rv = r4[t];
        xv.x += a * pv.x; xv.y += a * pv.y; xv.z += a * pv.z; xv.w += a * pv.w;
        rv.x -= a * qv.x; rv.y -= a * qv.y; rv.z -= a * qv.z; rv.w -= a * qv.w;
        x4[t] = xv;
        r4[t] = rv;
        acc[0] += ((double)rv.x * rv.x + (double)rv.y * rv.y) + ((double)rv.z * rv.z + (double)rv.w * rv.w);
    }
    for (long long t = 4 * n4 + bx * (long long)blockDim.x + threadIdx.x; t < cells; t += stride)
    {
        x[t] += a * p[t];
        const float rn = r[t] - a * q[t];
        r[t] = rn;
        acc[0] += (double)rn * rn;
    }
    GridReduceB<1>(R, acc, slotRR, (unsigned)bx, (unsigned)gx, 0, it);
}

// The same update on a colour-split level 0 with its tile activity (LevelView::act): the vector walked tile by tile
// (1024 elements of one colour's plane), the tiles that hold no unknown skipped (p and q are zero there, so x and r
// stay as they are and add nothing to r.r).
__device__ __forceinline__ void LinXRTiles(const LevelView &v, float *__restrict__ x, float *__restrict__ r,
                                           const float *p0, const float *p1, const float *__restrict__ q,
                                           const Reducer &R, const double *S, int *it, int baseEven, int baseOdd,
                                           int slotN, int singular, int slotPQ, int slotRR, int bx, int gx)
{
    const int par = *it & 1;
    const float *__restrict__ p = par ? p0 : p1;
    const int base = par ? baseOdd : baseEven;
    const float a = (float)(RzEffP(S, base, S[slotN], singular) / S[slotPQ]);
    double acc[1] = {0.0};
    const int tiles = v.actTiles, perColour = v.Ny * tiles, units = 2 * perColour;
    for (int u = bx; u < units; u += gx)
    {
        const int c = u / perColour, rem = u - c * perColour, i = rem / tiles, t = rem - i * tiles;
        if (!v.act[(long long)i * tiles + t]) continue;
        const long long e0 = (long long)c * v.sHalf + (long long)i * v.sPS + 4LL * kPairThreads * t;
        const int n4 = min(kPairThreads, (v.sPS - 4 * kPairThreads * t) >> 2);
        for (int k = threadIdx.x; k < n4; k += blockDim.x)
        {
            const long long o = e0 + 4LL * k;
            const float4 pv = *reinterpret_cast<const float4 *>(p + o), qv = *reinterpret_cast<const float4 *>(q + o);
            float4 xv = *reinterpret_cast<float4 *>(x + o), rv = *reinterpret_cast<float4 *>(r + o);
            xv.x += a * pv.x; xv.y += a * pv.y; xv.z += a * pv.z; xv.w += a * pv.w;
            rv.x -= a * qv.x; rv.y -= a * qv.y; rv.z -= a * qv.z; rv.w -= a * qv.w;
            *reinterpret_cast<float4 *>(x + o) = xv;
            *reinterpret_cast<float4 *>(r + o) = rv;
            acc[0] += ((double)rv.x * rv.x + (double)rv.y * rv.y) + ((double)rv.z * rv.z + (double)rv.w * rv.w);
        }
    }
    GridReduceB<1>(R, acc, slotRR, (unsigned)bx, (unsigned)gx, 0, it);
}

__global__ void __launch_bounds__(256) k_lin_xr_tiles(LevelView v, float *__restrict__ x, float *__restrict__ r,
                                                      const float *p0, const float *p1, const float *__restrict__ q,
                                                      Reducer R, const double *S, int *it, int baseEven, int baseOdd,
                                                      int slotN, int singular, int slotPQ, int slotRR)
{
    PdlWait();
    PdlTrigger();
    LinXRTiles(v, x, r, p0, p1, q, R, S, it, baseEven, baseOdd, slotN, singular, slotPQ, slotRR, (int)blockIdx.x,
               (int)gridDim.x);
}

__global__ void __launch_bounds__(256) k_lin_xr(long long cells, float *__restrict__ x, float *__restrict__ r,
                                                const float *p0, const float *p1, const float *__restrict__ q,
                                                Reducer R, const double *S, int *it, int baseEven, int baseOdd, int slotN,
                                                int singular, int slotPQ, int slotRR)
{
    PdlWait();
    PdlTrigger();
    LinXR(cells, x, r, p0, p1, q, R, S, it, baseEven, baseOdd, slotN, singular, slotPQ, slotRR, (int)blockIdx.x,
          (int)gridDim.x);
}

// batched (nb_batch.cu): block z runs the request at list[z]; r is its level 0's r
__global__ void __launch_bounds__(256) kb_lin_xr(const BatchLevel *__restrict__ lv, int ls,
                                                 const BatchReq *__restrict__ rq, BatchList a, int baseEven,
                                                 int baseOdd, int slotN, int slotPQ, int slotRR)
{
    PdlWait();
    PdlTrigger();
    const int q = BatchReqOf(a);
    if (q < 0) return;
    const BatchReq &Q = rq[q];
    const BatchLevel &L = lv[q * ls];
    if (L.v.act)
        LinXRTiles(L.v, Q.x, L.r, Q.p0, Q.p1, Q.q, Q.red, Q.red.out, Q.it, baseEven, baseOdd, slotN, Q.singular,
                   slotPQ, slotRR, (int)blockIdx.x, (int)gridDim.x);
    else
        LinXR(Q.vecLen, Q.x, L.r, Q.p0, Q.p1, Q.q, Q.red, Q.red.out, Q.it, baseEven, baseOdd, slotN, Q.singular,
              slotPQ, slotRR, (int)blockIdx.x, (int)gridDim.x);
}

void LaunchLinDot(long long cells, const float *r, const float *z, const Reducer &R, const int *it, int baseEven,
                  int baseOdd, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_lin_dot<<<kLinBlocks, 256, 0, st>>>(cells, r, z, R, it, baseEven, baseOdd);
}

void LaunchBatchLinXR(const BatchLevel *lv, int ls, const BatchReq *rq, BatchList a, int cap, int baseEven,
                      int baseOdd, int slotN, int slotPQ, int slotRR, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    LaunchPdl(kb_lin_xr, dim3(kLinBlocks, 1, cap), dim3(256), 0, st, lv, ls, rq, a, baseEven, baseOdd, slotN, slotPQ,
              slotRR);
}

void LaunchSplitLinXR(const LevelView &v, long long vecLen, float *x, float *r, const float *p0, const float *p1,
                      const float *q, const Reducer &R, const double *S, int *it, int baseEven, int baseOdd, int slotN,
                      int singular, int slotPQ, int slotRR, cudaStream_t st)
{
    if (!v.act)
    {
        LaunchLinXR(vecLen, x, r, p0, p1, q, R, S, it, baseEven, baseOdd, slotN, singular, slotPQ, slotRR, st);
        return;
    }
    NB_COUNT_LAUNCH();
    LaunchPdl(k_lin_xr_tiles, dim3(kLinBlocks), dim3(256), 0, st, v, x, r, p0, p1, q, R, S, it, baseEven, baseOdd,
              slotN, singular, slotPQ, slotRR);
}

void LaunchLinXR(long long cells, float *x, float *r, const float *p0, const float *p1, const float *q,
                 const Reducer &R, const double *S, int *it, int baseEven, int baseOdd, int slotN, int singular,
                 int slotPQ, int slotRR, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    LaunchPdl(k_lin_xr, dim3(kLinBlocks), dim3(256), 0, st, cells, x, r, p0, p1, q, R, S, it, baseEven, baseOdd, slotN,
              singular, slotPQ, slotRR);
}

} // namespace nb
