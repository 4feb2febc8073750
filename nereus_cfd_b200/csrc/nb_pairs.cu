// Multigrid and PCG kernels for 3D levels of a uniform grid in FP32 (the inner solve of the mixed-precision form),
// built for memory throughput.
//
// Cell pairs. With Nz even, the two cells (i, j, 2m) and (i, j, 2m+1) form an 8-byte aligned pair, and a plane of
// Nx*Nz cells is Nx*Nz/2 consecutive pairs. Thread t of the launch takes pair t of the plane (crossing row ends
// freely: a row's ring cells ride along, their vector entries are zero) and marches along i over kPairS planes,
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

namespace nb
{

namespace
{

constexpr int kPairThreads = 256;
constexpr int kPairS = 8; // planes a thread marches

// Per-thread position of a pair kernel.
struct PairPos
{
    int lane;
    bool valid;  // false for the clamped threads past the plane's last pair (they still load and shuffle)
    int i0, i1;  // planes [i0, i1)
    int sI, sJ;
    int j, k0;   // row and first cell of the pair (k0 even)
    long long base; // cell index of the pair's first cell on plane i0
};

__device__ __forceinline__ PairPos PairStart(const LevelView &v)
{
    PairPos p;
    const int P = (int)(v.sI >> 1);
    p.lane = threadIdx.x & 31;
    int q = blockIdx.x * kPairThreads + threadIdx.x;
    p.valid = q < P;
    if (!p.valid) q = P - 1;
    p.i0 = 1 + blockIdx.y * kPairS;
    p.i1 = min(p.i0 + kPairS, v.Ny - 1);
    p.sI = (int)v.sI;
    p.sJ = (int)v.sJ;
    const int cin = 2 * q;
    p.j = cin / v.Nz;
    p.k0 = cin - p.j * v.Nz;
    p.base = (long long)p.i0 * v.sI + cin;
    return p;
}

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
        if (!interior || v.types[c] != FLUID) { du[c] = 0; continue; }
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
        du[c] = (uint8_t)(0x80u | units);
    }
}

bool PairLevelShape(const LevelView &v) { return v.dim == 3 && !v.stretched && (v.Nz % 2) == 0 && v.Ny >= 3; }

void LaunchBuildDu(const LevelView &v, uint8_t *du, cudaStream_t st)
{
    int blocks = (int)((v.cells + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    NB_COUNT_LAUNCH();
    k_build_du<<<blocks, 256, 0, st>>>(v, du);
}

static inline dim3 PairGrid(const LevelView &v)
{
    const long long P = v.sI / 2;
    return dim3((unsigned)((P + kPairThreads - 1) / kPairThreads), (unsigned)((v.Ny - 2 + kPairS - 1) / kPairS));
}

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
// read has the other colour, so nothing read changes during the sweep.
__global__ void __launch_bounds__(kPairThreads) k_pair_half(LevelView v, const uint8_t *__restrict__ du,
                                                            const float *__restrict__ r, float *e, int colour)
{
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
        if (P.valid) ep[off + (second ? 1 : 0)] = (rv + g * s) * inv[units];
        eM = eC;
        eC = eP;
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

void LaunchPairFirst(const LevelView &v, const uint8_t *du, const float *r, float *e, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_pair_first<<<PairGrid(v), kPairThreads, 0, st>>>(v, du, r, e);
}

void LaunchPairHalf(const LevelView &v, const uint8_t *du, const float *r, float *e, int colour, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_pair_half<<<PairGrid(v), kPairThreads, 0, st>>>(v, du, r, e, colour);
}

void LaunchPairResidual(const LevelView &v, const uint8_t *du, const float *r, const float *e, float *res,
                        cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_pair_residual<<<PairGrid(v), kPairThreads, 0, st>>>(v, du, r, e, res);
}

// ---------------------------------------------------------------------------------------------------------------
// PCG on level 0 (the semantics of k_update_p_apply / k_dot / k_update_xr in nb_kernels.cu)
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ double RzEffP(const double *S, int base, int n, int singular)
{
    return singular ? S[base] - (S[base + 1] / (double)n) * S[base + 2] : S[base];
}

// p_new = U (z - mean + beta p_old), q = M p_new, sum p_new.q; U = 1 on unknowns (needed only when the mean of z is
// removed: elsewhere z and p_old are zero already).
template <bool kSingular>
__global__ void __launch_bounds__(kPairThreads)
    k_pair_papply(LevelView v, const uint8_t *__restrict__ du, const float *__restrict__ z, float *p0, float *p1,
                  float *__restrict__ q, Reducer R, const double *S, const int *it, int baseEven, int baseOdd, int n,
                  int slotPQ)
{
    const int iter = *it, par = iter & 1;
    const float *__restrict__ pIn = par ? p1 : p0;
    float *__restrict__ pOut = par ? p0 : p1;
    const int baseNew = par ? baseOdd : baseEven, baseOld = par ? baseEven : baseOdd;
    const double beta = iter == 0 ? 0.0 : RzEffP(S, baseNew, n, kSingular) / RzEffP(S, baseOld, n, kSingular);
    const float b = (float)beta;
    const float mean = kSingular ? (float)(S[baseNew + 1] / (double)n) : 0.f;
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
    double acc[1] = {0.0};
    int off = 0;
    for (int i = P.i0; i < P.i1; i++, off += P.sI)
    {
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
        qq.x = Unk(d) * (hg * (float)(d & 0x7Fu) * NC.x - g * s0);
        qq.y = Unk(d >> 8) * (hg * (float)((d >> 8) & 0x7Fu) * NC.y - g * s1);
        if (P.valid)
        {
            *reinterpret_cast<float2 *>(pOut + P.base + off) = NC;
            *reinterpret_cast<float2 *>(q + P.base + off) = qq;
            acc[0] += (double)NC.x * (double)qq.x + (double)NC.y * (double)qq.y;
        }
        NM = NC;
        NC = NP;
    }
    GridReduce<1>(R, acc, slotPQ);
}

void LaunchPairPApply(const LevelView &v, const uint8_t *du, const float *z, float *p0, float *p1, float *q,
                      const Reducer &R, const double *S, const int *it, int baseEven, int baseOdd, int n,
                      int singular, int slotPQ, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    if (singular)
        k_pair_papply<true><<<PairGrid(v), kPairThreads, 0, st>>>(v, du, z, p0, p1, q, R, S, it, baseEven, baseOdd,
                                                                   n, slotPQ);
    else
        k_pair_papply<false><<<PairGrid(v), kPairThreads, 0, st>>>(v, du, z, p0, p1, q, R, S, it, baseEven, baseOdd,
                                                                    n, slotPQ);
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
__global__ void __launch_bounds__(256) k_lin_xr(long long cells, float *__restrict__ x, float *__restrict__ r,
                                                const float *p0, const float *p1, const float *__restrict__ q,
                                                Reducer R, const double *S, int *it, int baseEven, int baseOdd, int n,
                                                int singular, int slotPQ, int slotRR)
{
    const int par = *it & 1;
    const float *__restrict__ p = par ? p0 : p1;
    const int base = par ? baseOdd : baseEven;
    const float a = (float)(RzEffP(S, base, n, singular) / S[slotPQ]);
    double acc[1] = {0.0};
    const long long n4 = cells >> 2, stride = (long long)gridDim.x * blockDim.x;
    float4 *x4 = reinterpret_cast<float4 *>(x), *r4 = reinterpret_cast<float4 *>(r);
    const float4 *p4 = reinterpret_cast<const float4 *>(p), *q4 = reinterpret_cast<const float4 *>(q);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n4; t += stride)
    {
        const float4 pv = p4[t], qv = q4[t];
        float4 xv = x4[t], rv = r4[t];
        xv.x += a * pv.x; xv.y += a * pv.y; xv.z += a * pv.z; xv.w += a * pv.w;
        rv.x -= a * qv.x; rv.y -= a * qv.y; rv.z -= a * qv.z; rv.w -= a * qv.w;
        x4[t] = xv;
        r4[t] = rv;
        acc[0] += ((double)rv.x * rv.x + (double)rv.y * rv.y) + ((double)rv.z * rv.z + (double)rv.w * rv.w);
    }
    for (long long t = 4 * n4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cells; t += stride)
    {
        x[t] += a * p[t];
        const float rn = r[t] - a * q[t];
        r[t] = rn;
        acc[0] += (double)rn * rn;
    }
    GridReduce<1>(R, acc, slotRR, 0, it);
}

void LaunchLinDot(long long cells, const float *r, const float *z, const Reducer &R, const int *it, int baseEven,
                  int baseOdd, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_lin_dot<<<kLinBlocks, 256, 0, st>>>(cells, r, z, R, it, baseEven, baseOdd);
}

void LaunchLinXR(long long cells, float *x, float *r, const float *p0, const float *p1, const float *q,
                 const Reducer &R, const double *S, int *it, int baseEven, int baseOdd, int n, int singular,
                 int slotPQ, int slotRR, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_lin_xr<<<kLinBlocks, 256, 0, st>>>(cells, x, r, p0, p1, q, R, S, it, baseEven, baseOdd, n, singular, slotPQ,
                                         slotRR);
}

} // namespace nb
