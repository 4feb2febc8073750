// Multigrid and PCG kernels for 3D FP32 levels in the colour-split layout (the inner solve of the mixed-precision
// form), built so that each red-black half-sweep moves only the bytes the algorithm needs.
//
// Colour-split layout. Cell (i, j, k) has colour c = (i + j + k) & 1 and sits at c*H + i*PS + j*RS + (k >> 1) of a
// level vector: each colour is an Ny x Nx x RS array whose rows hold the Nz/2 cells of that colour (RS = Nz/2
// rounded up to 4, the padding kept at zero). In row (i, j) the cell of colour c at element m is k = 2m + q with
// q = (i + j + c) & 1, and its six neighbours all have the other colour:
//   (i +- 1, j, m), (i, j +- 1, m), (i, j, m) and (i, j, m + (q ? 1 : -1)).
// A half-sweep of colour c therefore reads the other colour, r and the diagonal bytes of colour c, and writes
// colour c: half of every array, where a cell-pair sweep reads and writes both colours.
//
// Quads. Thread t of a launch takes the four elements 4t .. 4t+3 of a plane of one colour (RS is a multiple of 4, so
// a quad never crosses a row) and marches along i over up to kPairS planes, keeping planes i-1, i, i+1 in
// registers. The j neighbours are the quads RS elements away; the element across the quad's edge comes from the
// neighbouring lane (a shuffle; lanes 0 and 31 load it).
//
// Every vector is zero off the unknowns (and on the padding), so the neighbour sum runs over all six neighbours. The
// levels are uniform (a stretched grid keeps the cell-pair kernels of nb_pairs.cu): the coefficient is gamma
// everywhere and the diagonal is gamma/2 times the unit count in the level's byte array (0x80 | units, 0 off the
// unknowns), divided through a 32-entry reciprocal table.
//
// The V-cycle on these levels (nb_solver.cu, VCycleSplit) uses two facts of red-black Gauss-Seidel:
// - after a black half-sweep the black residual is zero (each black equation was just solved), so the residual and
//   its restriction run over the red cells only;
// - a black half-sweep does not read the black values it replaces, so the prolonged coarse correction is added to
//   the red cells only before the post-smoothing, which starts black.
#include "nb_kernels.h"

namespace nb
{

namespace
{

struct F4
{
    float v[4];
};

__device__ __forceinline__ F4 L4(const float *p)
{
    const float4 a = *reinterpret_cast<const float4 *>(p);
    return F4{{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ void S4(float *p, const F4 &a)
{
    *reinterpret_cast<float4 *>(p) = make_float4(a.v[0], a.v[1], a.v[2], a.v[3]);
}
__device__ __forceinline__ unsigned LdU4(const uint8_t *p) { return *reinterpret_cast<const unsigned *>(p); }
// loads of values a kernel reads once (evict-first): measured to keep the half-sweep's j-row loads in L1 longer
__device__ __forceinline__ F4 L4Once(const float *p)
{
    const float4 a = __ldcs(reinterpret_cast<const float4 *>(p));
    return F4{{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ unsigned LdU4Once(const uint8_t *p) { return __ldcs(reinterpret_cast<const unsigned *>(p)); }
__device__ __forceinline__ unsigned Byte(unsigned d, int x) { return (d >> (8 * x)) & 0xFFu; }
__device__ __forceinline__ float Unk(unsigned b) { return (b & 0x80u) ? 1.0f : 0.0f; }

// 1 / (gamma/2 * units), entry 0 = 0
__device__ __forceinline__ void FillInv(float *inv, double gamma)
{
    if (threadIdx.x < 32) inv[threadIdx.x] = threadIdx.x ? 1.0f / (0.5f * (float)gamma * (float)threadIdx.x) : 0.0f;
    __syncthreads();
}

// Per-thread position of a quad kernel.
struct QuadPos
{
    int lane;
    bool valid;  // false for the clamped threads past the plane's last quad (they still load and shuffle)
    int i0, i1;  // planes [i0, i1)
    int j, m0;   // row and first element of the quad
    int RS, PS;
    long long off; // element of the quad on plane i0, within one colour
};

__device__ __forceinline__ QuadPos QuadStart(const LevelView &v, const Blk &b)
{
    QuadPos p;
    const int Q = v.sRS >> 2, nq = v.Nx * Q;
    p.lane = threadIdx.x & 31;
    int t = b.x * kPairThreads + threadIdx.x;
    p.valid = t < nq;
    if (!p.valid) t = nq - 1;
    // grid.y splits the Ny-2 interior planes into chunks of S (the host sized it); a block past the last plane starts
    // at the ring plane and marches none
    const int S = (v.Ny - 2 + b.gy - 1) / b.gy;
    p.i0 = min(1 + b.y * S, v.Ny - 1);
    p.i1 = min(p.i0 + S, v.Ny - 1);
    p.RS = v.sRS;
    p.PS = v.sPS;
    p.j = t / Q;
    p.m0 = 4 * (t - p.j * Q);
    p.off = (long long)p.i0 * v.sPS + 4LL * t;
    return p;
}

// True when no tile this block owns on planes [i0, i1) holds an unknown (LevelView::act): the block's cells are
// all zero in every vector and stay so, so it has nothing to compute, load or store.
__device__ __forceinline__ bool TileIdle(const LevelView &v, int bx, int i0, int i1)
{
    if (!v.act) return false;
    for (int i = i0; i < i1; i++)
        if (v.act[(long long)i * v.actTiles + bx]) return false;
    return true;
}

// The same for a block of a grid-layout pair kernel (PairStart): its rows j0 .. j1 of planes [i0, i1), checked
// through the split tiles that hold those rows' cells in either colour.
__device__ __forceinline__ bool RowsIdle(const LevelView &v, int j0, int j1, int i0, int i1)
{
    if (!v.act) return false;
    const int t0 = (int)(((long long)j0 * v.sRS) / (4 * kPairThreads));
    const int t1 = min(v.actTiles - 1, (int)(((long long)(j1 + 1) * v.sRS - 1) / (4 * kPairThreads)));
    for (int i = i0; i < i1; i++)
        for (int t = t0; t <= t1; t++)
            if (v.act[(long long)i * v.actTiles + t]) return false;
    return true;
}

// Resident blocks of a kernel per SM at kPairThreads threads (its registers and shared memory decide), and the SM
// count of the current device.
inline int ResidentBlocks(const void *fn)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kPairThreads, 0) != cudaSuccess || n < 1) n = 1;
    return n;
}

// read once per kernel (and before any stream capture: PrepareSplitKernels)
template <auto kKernel> int Occ()
{
    static const int n = ResidentBlocks((const void *)kKernel);
    return n;
}

inline int SmCount()
{
    int d = 0, c = 0;
    if (cudaGetDevice(&d) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, d) != cudaSuccess || c < 1) c = 148;
    return c;
}

// The launch grid of a quad kernel with `resident` blocks per SM: the longest march (planes per thread, at most
// kQuadMaxS) whose launch fills the last wave of resident blocks to at least 90%; the longer the march, the fewer
// planes of a neighbour array are loaded twice (a chunk of S planes loads S + 2). Measured on a 258^3 level: one
// 92%-full wave of 16-plane chunks beats two waves of 8 (and 1.03 waves of 15 runs at half speed). With no such S,
// the best-filled one (a small level fills no wave: S = 1, all the parallelism there is).
constexpr int kQuadMaxS = 16;

// The march length S (planes per thread, 1 .. kQuadMaxS) for a grid of perPlane x ceil(planes / S) blocks on `slots`
// resident blocks, by the rule above.
inline long long BestMarch(long long perPlane, long long planes, long long slots)
{
    long long bestS = 1;
    double bestU = -1.0;
    for (long long S = kQuadMaxS; S >= 1; S--)
    {
        const long long blocks = perPlane * ((planes + S - 1) / S);
        const long long waves = (blocks + slots - 1) / slots;
        const double u = (double)blocks / (double)(waves * slots);
        if (u >= 0.9) return S;
        if (u > bestU + 1e-9)
        {
            bestU = u;
            bestS = S;
        }
    }
    return bestS;
}

// A quad kernel's grid with a march of S planes (S > 0), or sized as above (S = 0).
inline dim3 QuadGridS(const LevelView &v, int S)
{
    const long long nq = (long long)v.Nx * (v.sRS / 4), perPlane = (nq + kPairThreads - 1) / kPairThreads;
    const long long planes = v.Ny - 2 > 0 ? v.Ny - 2 : 1;
    return dim3((unsigned)perPlane, (unsigned)((planes + S - 1) / S));
}

inline dim3 QuadGrid(const LevelView &v, int resident)
{
    const long long nq = (long long)v.Nx * (v.sRS / 4), perPlane = (nq + kPairThreads - 1) / kPairThreads;
    const long long planes = v.Ny - 2 > 0 ? v.Ny - 2 : 1;
    const long long bestS = BestMarch(perPlane, planes, (long long)SmCount() * (resident > 0 ? resident : 1));
    return dim3((unsigned)perPlane, (unsigned)((planes + bestS - 1) / bestS));
}

// The other colour's k neighbours of a quad: the element at m (c) and the one at m + (q ? 1 : -1) (returned).
__device__ __forceinline__ F4 KShift(const F4 &c, float prevW, float nextX, int q)
{
    return q ? F4{{c.v[1], c.v[2], c.v[3], nextX}} : F4{{prevW, c.v[0], c.v[1], c.v[2]}};
}

// The elements just before and after this lane's quad in its row (0 past the row's ends; the values a lane takes
// from a neighbouring row only reach ring or padding cells, whose results are masked).
__device__ __forceinline__ void Edges(const QuadPos &P, const F4 &c, const float *row, float &prevW, float &nextX)
{
    prevW = __shfl_up_sync(0xffffffffu, c.v[3], 1);
    nextX = __shfl_down_sync(0xffffffffu, c.v[0], 1);
    if (P.lane == 0) prevW = P.m0 > 0 ? row[-1] : 0.f;
    if (P.lane == 31) nextX = P.m0 + 4 < P.RS ? row[4] : 0.f;
}

} // namespace

// planes per thread at least in the pair-thread launches that end in a grid-wide sum
constexpr int kSplitReduceS = 16;

// ---------------------------------------------------------------------------------------------------------------
// smoothing
// ---------------------------------------------------------------------------------------------------------------

// The first red-black sweep from a zero iterate on a uniform level, one launch: red e = r / diag, then black
// e = (r + gamma * sum of the red neighbours) / diag with the red neighbours formed from r and the bytes. A thread
// owns one quad position and writes the red and the black quad there.
__device__ __forceinline__ void SplitFirst(const LevelView &v, const uint8_t *__restrict__ du,
                                           const float *__restrict__ r, float *__restrict__ e, const Blk &blk)
{
    __shared__ float inv[32];
    FillInv(inv, v.gamma);
    const QuadPos P = QuadStart(v, blk);
    if (TileIdle(v, blk.x, P.i0, P.i1)) return;
    const float g = (float)v.gamma;
    const long long hb = v.sHalf;
    const float *R0 = r + P.off, *R1 = r + hb + P.off;
    const uint8_t *D0 = du + P.off, *D1 = du + hb + P.off;
    float *X0 = e + P.off, *X1 = e + hb + P.off;
    auto red = [&](long long o) {
        F4 a = L4(R0 + o);
        const unsigned d = LdU4(D0 + o);
#pragma unroll
        for (int x = 0; x < 4; x++) a.v[x] *= inv[Byte(d, x) & 0x7Fu];
        return a;
    };
    auto red1 = [&](long long o) { return R0[o] * inv[D0[o] & 0x7Fu]; };
    F4 RM = red(-P.PS), RC = red(0);
    long long o = 0;
    for (int i = P.i0; i < P.i1; i++, o += P.PS)
    {
        const F4 RP = red(o + P.PS), RJp = red(o + P.RS), RJm = red(o - P.RS);
        const F4 rb = L4Once(R1 + o);
        const unsigned db = LdU4Once(D1 + o);
        float prevW = __shfl_up_sync(0xffffffffu, RC.v[3], 1), nextX = __shfl_down_sync(0xffffffffu, RC.v[0], 1);
        if (P.lane == 0) prevW = P.m0 > 0 ? red1(o - 1) : 0.f;
        if (P.lane == 31) nextX = P.m0 + 4 < P.RS ? red1(o + 4) : 0.f;
        const F4 sh = KShift(RC, prevW, nextX, (i + P.j + 1) & 1);
        F4 nb;
#pragma unroll
        for (int x = 0; x < 4; x++)
        {
            const float s = ((RP.v[x] + RM.v[x]) + (RJp.v[x] + RJm.v[x])) + (RC.v[x] + sh.v[x]);
            nb.v[x] = (rb.v[x] + g * s) * inv[Byte(db, x) & 0x7Fu];
        }
        if (P.valid)
        {
            S4(X0 + o, RC);
            S4(X1 + o, nb);
        }
        RM = RC;
        RC = RP;
    }
}

__global__ void __launch_bounds__(kPairThreads) k_split_first(LevelView v, const uint8_t *__restrict__ du,
                                                              const float *__restrict__ r, float *__restrict__ e)
{
    PdlWait();
    PdlTrigger();
    SplitFirst(v, du, r, e, ThisBlk());
}

// One colour of a red-black sweep: e_c = (r_c + gamma * sum of the other colour's six neighbours) / diag_c.
// kDot 1: (sum r.e, sum e, sum r) of this colour into out[partSlot..]; kDot 2: the same plus the totals already in
// out[partSlot..], into the scalar block of the iteration's parity (the CG's r.z, sum z, sum r of the V-cycle's z).
// du, r: this colour's halves; eo, ec: the other colour's and this colour's halves of e (disjoint).
template <int kDot>
__device__ __forceinline__ void SplitHalf(const LevelView &v, const uint8_t *__restrict__ du,
                                          const float *__restrict__ r, const float *__restrict__ eo,
                                          float *__restrict__ ec, int colour, const Reducer &R, const int *it,
                                          int baseEven, int baseOdd, int partSlot, const Blk &blk)
{
    float facc[3] = {0.f, 0.f, 0.f}; // a thread's terms in FP32, the block and grid sums in FP64
    __shared__ float inv[32];
    FillInv(inv, v.gamma);
    QuadPos P = QuadStart(v, blk);
    if (TileIdle(v, blk.x, P.i0, P.i1))
    {
        if (!kDot) return;
        P.i1 = P.i0; // nothing to sweep; the block still adds its zero terms to the sums
    }
    const float g = (float)v.gamma;
    const float *O = eo + P.off;
    const float *Rr = r + P.off;
    const uint8_t *D = du + P.off;
    float *C = ec + P.off;
    // one plane: the six other-colour neighbours, r and the bytes given, the new values stored (and summed)
    auto plane = [&](int i, long long o, const F4 &oM, const F4 &oC, const F4 &oP, const F4 &jp, const F4 &jm,
                     const F4 &rr, unsigned d) {
        float prevW, nextX;
        Edges(P, oC, O + o, prevW, nextX);
        const F4 sh = KShift(oC, prevW, nextX, (i + P.j + colour) & 1);
        F4 nv;
#pragma unroll
        for (int x = 0; x < 4; x++)
        {
            const float s = ((oP.v[x] + oM.v[x]) + (jp.v[x] + jm.v[x])) + (oC.v[x] + sh.v[x]);
            nv.v[x] = (rr.v[x] + g * s) * inv[Byte(d, x) & 0x7Fu];
        }
        if (P.valid)
        {
            S4(C + o, nv);
            if (kDot)
            {
#pragma unroll
                for (int x = 0; x < 4; x++)
                {
                    facc[0] += rr.v[x] * nv.v[x];
                    facc[1] += nv.v[x];
                    facc[2] += rr.v[x];
                }
            }
        }
    };
    // two planes per trip: all the streamed values of both (the other colour up to two planes ahead, the j rows,
    // r and the bytes) are loaded before either is computed, twice the loads in flight of a plane-by-plane march
    F4 oM{}, oC{};
    if (P.i0 < P.i1)
    {
        oM = L4(O - P.PS);
        oC = L4(O);
    }
    long long o = 0;
    for (int i = P.i0; i < P.i1; i += 2, o += 2 * P.PS)
    {
        const bool two = i + 1 < P.i1;
        const F4 oP = L4(O + o + P.PS);
        const F4 oPP = two ? L4(O + o + 2 * P.PS) : F4{};
        const F4 r0 = L4Once(Rr + o), r1 = two ? L4Once(Rr + o + P.PS) : F4{};
        const unsigned d0 = LdU4Once(D + o), d1 = two ? LdU4Once(D + o + P.PS) : 0u;
        const F4 jp0 = L4(O + o + P.RS), jm0 = L4(O + o - P.RS);
        const F4 jp1 = two ? L4(O + o + P.PS + P.RS) : F4{}, jm1 = two ? L4(O + o + P.PS - P.RS) : F4{};
        plane(i, o, oM, oC, oP, jp0, jm0, r0, d0);
        if (two) plane(i + 1, o + P.PS, oC, oP, oPP, jp1, jm1, r1, d1);
        oM = oP;
        oC = oPP;
    }
    if (kDot == 1)
    {
        double acc[3] = {facc[0], facc[1], facc[2]};
        GridReduceB<3>(R, acc, partSlot, BlkId(blk), BlkCount(blk));
    }
    else if (kDot == 2)
    {
        double acc[3] = {facc[0], facc[1], facc[2]};
        GridReduceB<3>(R, acc, (*it & 1) ? baseOdd : baseEven, BlkId(blk), BlkCount(blk), 0, nullptr, partSlot);
    }
}

// 4 resident blocks (64 registers): the two-plane march measured 12% faster there than at 3 (73 registers)
template <int kDot>
__global__ void __launch_bounds__(kPairThreads, 4)
    k_split_half(LevelView v, const uint8_t *__restrict__ du, const float *__restrict__ r,
                 const float *__restrict__ eo, float *__restrict__ ec, int colour, Reducer R, const int *it,
                 int baseEven, int baseOdd, int partSlot)
{
    PdlWait();
    PdlTrigger();
    SplitHalf<kDot>(v, du, r, eo, ec, colour, R, it, baseEven, baseOdd, partSlot, ThisBlk());
}

// the arguments of k_split_half for colour c: its halves of du and r, the other colour's and its own halves of e
#define NB_SPLIT_HALF_ARGS(c)                                                                                      \
    v, du + (long long)(c) * v.sHalf, r + (long long)(c) * v.sHalf, e + (long long)((c) ^ 1) * v.sHalf,               \
        e + (long long)(c) * v.sHalf, (c)

void LaunchSplitFirst(const LevelView &v, const uint8_t *du, const float *r, float *e, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    LaunchPdl(k_split_first, QuadGrid(v, Occ<k_split_first>()), kPairThreads, 0, st, v, du, r, e);
}

void LaunchSplitHalf(const LevelView &v, const uint8_t *du, const float *r, float *e, int colour, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    LaunchPdl(k_split_half<0>, QuadGrid(v, Occ<k_split_half<0>>()), kPairThreads, 0, st, NB_SPLIT_HALF_ARGS(colour),
              Reducer{}, (const int *)nullptr, 0, 0, 0);
}

void LaunchSplitHalfDot(const LevelView &v, const uint8_t *du, const float *r, float *e, int colour, bool last,
                        const Reducer &R, const int *it, int baseEven, int baseOdd, int partSlot, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    if (last)
        LaunchPdl(k_split_half<2>, QuadGrid(v, Occ<k_split_half<2>>()), kPairThreads, 0, st,
                  NB_SPLIT_HALF_ARGS(colour), R, it, baseEven, baseOdd, partSlot);
    else
        LaunchPdl(k_split_half<1>, QuadGrid(v, Occ<k_split_half<1>>()), kPairThreads, 0, st,
                  NB_SPLIT_HALF_ARGS(colour), R, it, baseEven, baseOdd, partSlot);
}
#undef NB_SPLIT_HALF_ARGS

// res = r - M e on the red cells (colour 0), into the first half of `res`; the black residual after a black
// half-sweep is zero.
__device__ __forceinline__ void SplitResidual(const LevelView &v, const uint8_t *__restrict__ du,
                                              const float *__restrict__ r, const float *__restrict__ e,
                                              float *__restrict__ res, const Blk &blk)
{
    const QuadPos P = QuadStart(v, blk);
    if (TileIdle(v, blk.x, P.i0, P.i1)) return;
    const float g = (float)v.gamma, hg = 0.5f * (float)v.gamma;
    const float *O = e + v.sHalf + P.off;
    const float *Xr = e + P.off;
    const float *Rr = r + P.off;
    const uint8_t *D = du + P.off;
    float *Out = res + P.off;
    auto plane = [&](int i, long long o, const F4 &oM, const F4 &oC, const F4 &oP, const F4 &jp, const F4 &jm,
                     const F4 &xc, const F4 &rr, unsigned d) {
        float prevW, nextX;
        Edges(P, oC, O + o, prevW, nextX);
        const F4 sh = KShift(oC, prevW, nextX, (i + P.j) & 1);
        F4 out;
#pragma unroll
        for (int x = 0; x < 4; x++)
        {
            const unsigned b = Byte(d, x);
            const float s = ((oP.v[x] + oM.v[x]) + (jp.v[x] + jm.v[x])) + (oC.v[x] + sh.v[x]);
            out.v[x] = (b & 0x80u) ? rr.v[x] - (hg * (float)(b & 0x7Fu) * xc.v[x] - g * s) : 0.f;
        }
        if (P.valid) S4(Out + o, out);
    };
    // two planes per trip, all their streamed values loaded first (as in the half-sweep)
    F4 oM = L4(O - P.PS), oC = L4(O);
    long long o = 0;
    for (int i = P.i0; i < P.i1; i += 2, o += 2 * P.PS)
    {
        const bool two = i + 1 < P.i1;
        const F4 oP = L4(O + o + P.PS), oPP = two ? L4(O + o + 2 * P.PS) : F4{};
        const F4 jp0 = L4(O + o + P.RS), jm0 = L4(O + o - P.RS);
        const F4 jp1 = two ? L4(O + o + P.PS + P.RS) : F4{}, jm1 = two ? L4(O + o + P.PS - P.RS) : F4{};
        const F4 x0 = L4(Xr + o), r0 = L4Once(Rr + o), x1 = two ? L4(Xr + o + P.PS) : F4{},
                 r1 = two ? L4Once(Rr + o + P.PS) : F4{};
        const unsigned d0 = LdU4Once(D + o), d1 = two ? LdU4Once(D + o + P.PS) : 0u;
        plane(i, o, oM, oC, oP, jp0, jm0, x0, r0, d0);
        if (two) plane(i + 1, o + P.PS, oC, oP, oPP, jp1, jm1, x1, r1, d1);
        oM = oP;
        oC = oPP;
    }
}

__global__ void __launch_bounds__(kPairThreads, 4) k_split_residual(LevelView v, const uint8_t *__restrict__ du,
                                                                 const float *__restrict__ r,
                                                                 const float *__restrict__ e, float *__restrict__ res)
{
    PdlWait();
    PdlTrigger();
    SplitResidual(v, du, r, e, res, ThisBlk());
}

void LaunchSplitResidual(const LevelView &v, const uint8_t *du, const float *r, const float *e, float *res,
                         cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    LaunchPdl(k_split_residual, QuadGrid(v, Occ<k_split_residual>()), kPairThreads, 0, st, v, du, r, e, res);
}

// ---------------------------------------------------------------------------------------------------------------
// transfers between a split level and the next coarser level (either layout): the operators of k_prolong and
// k_restrict on the red cells
// ---------------------------------------------------------------------------------------------------------------
// Per red fine cell (colour-split, red half only): 0x80 for an unknown, plus in the low six bits the weight (in 1/64)
// that the Neumann-aware prolongation moves from the cell's SOLID coarse contributors onto its parent.

// e_f += P e_c on the red fine unknowns. Fine k = 2m + q (q = (a + b) & 1) lies between coarse k-cells m and m+1
// with weights (3/4, 1/4) for q = 0 and (1/4, 3/4) for q = 1; its parent is m + q. Fine row 2B-1 mixes coarse rows
// B (3/4) and B-1 (1/4), row 2B rows B and B+1; planes the same way.
//
// A thread owns coarse row B and the fine quad m0 .. m0+3 of fine rows 2B-1 and 2B, and marches along the coarse
// planes A: per coarse plane it interpolates three coarse rows across j once (k-cells m0 .. m0+4), and with the
// neighbouring planes' rows (kept in registers) serves the four fine quads of fine planes 2A-1, 2A and rows 2B-1,
// 2B, whose red values and bytes it loads together.

// coarse k-cells m0 .. m0+4 of coarse row (A, B)
__device__ __forceinline__ void CoarseRow5(const LevelView &cv, const float *__restrict__ ec, int A, int B, int m0,
                                           float c[5])
{
    const int Dmax = cv.Nz - 1;
    if (cv.sRS && m0 + 4 <= Dmax)
    {
        // a colour-split coarse level: k-cells m0, m0+2, m0+4 are elements m0/2 .. m0/2+2 of colour (A+B) & 1, and
        // m0+1, m0+3 elements m0/2, m0/2+1 of the other (m0 is a multiple of 4)
        const int ce = (A + B) & 1;
        const float *rb = ec + (long long)A * cv.sPS + (long long)B * cv.sRS + (m0 >> 1);
        const float2 ev = *reinterpret_cast<const float2 *>(rb + ce * cv.sHalf);
        const float2 od = *reinterpret_cast<const float2 *>(rb + (ce ^ 1) * cv.sHalf);
        c[0] = ev.x;
        c[1] = od.x;
        c[2] = ev.y;
        c[3] = od.y;
        c[4] = rb[ce * cv.sHalf + 2];
        return;
    }
#pragma unroll
    for (int t = 0; t < 5; t++) c[t] = ec[VecIdx(cv, A, B, min(m0 + t, Dmax))]; // past the row: masked cells only
}

// the coarse plane's rows interpolated across j for fine rows 2B-1 (y0) and 2B (y1), and row B itself (par)
__device__ __forceinline__ void CoarsePlaneRows(const LevelView &cv, const float *__restrict__ ec, int A, int B,
                                                int m0, float y0[5], float y1[5], float par[5])
{
    float cm[5], cp[5];
    CoarseRow5(cv, ec, A, B, m0, par);
    CoarseRow5(cv, ec, A, B - 1, m0, cm);
    CoarseRow5(cv, ec, A, B + 1, m0, cp);
#pragma unroll
    for (int t = 0; t < 5; t++)
    {
        y0[t] = 0.75f * par[t] + 0.25f * cm[t];
        y1[t] = 0.75f * par[t] + 0.25f * cp[t];
    }
}

__device__ __forceinline__ void SplitProlong(const LevelView &fv, const LevelView &cv,
                                             const uint8_t *__restrict__ pext, const float *__restrict__ ec,
                                             float *__restrict__ ef, const Blk &blk)
{
    const int Q = fv.sRS >> 2, nrow = cv.Nx - 2, nq = nrow * Q;
    int t = blk.x * kPairThreads + threadIdx.x;
    const bool valid = t < nq;
    if (!valid) t = nq - 1;
    const int B = 1 + t / Q, m0 = 4 * (t - (B - 1) * Q);
    const int S = (cv.Ny - 2 + blk.gy - 1) / blk.gy;
    const int A0 = min(1 + blk.y * S, cv.Ny - 1), A1 = min(A0 + S, cv.Ny - 1);
    if (!valid || A0 >= A1) return;
    float yM0[5], yM1[5], yC0[5], yC1[5], pC[5], pD[5];
    CoarsePlaneRows(cv, ec, A0 - 1, B, m0, yM0, yM1, pD);
    CoarsePlaneRows(cv, ec, A0, B, m0, yC0, yC1, pC);
    const int fb0 = 2 * B - 1, fb1 = 2 * B;
    for (int A = A0; A < A1; A++)
    {
        float yP0[5], yP1[5], pP[5];
        CoarsePlaneRows(cv, ec, A + 1, B, m0, yP0, yP1, pP);
        // fine planes 2A-1 (with coarse plane A-1) and 2A (with A+1), rows 2B-1 and 2B
#pragma unroll
        for (int h = 0; h < 2; h++)
        {
            const int fa = 2 * A - 1 + h;
            const long long o0 = (long long)fa * fv.sPS + (long long)fb0 * fv.sRS + m0, o1 = o0 + fv.sRS;
            const unsigned w0 = LdU4(pext + o0), w1 = LdU4(pext + o1);
            F4 e0 = L4(ef + o0), e1 = L4(ef + o1);
            const float *yo0 = h ? yP0 : yM0, *yo1 = h ? yP1 : yM1;
#pragma unroll
            for (int rI = 0; rI < 2; rI++)
            {
                const unsigned w = rI ? w1 : w0;
                if (!(w & 0x80808080u)) continue;
                const int q = (fa + (rI ? fb1 : fb0)) & 1;
                float z[5];
#pragma unroll
                for (int k = 0; k < 5; k++)
                    z[k] = rI ? 0.75f * yC1[k] + 0.25f * yo1[k] : 0.75f * yC0[k] + 0.25f * yo0[k];
                F4 &ev = rI ? e1 : e0;
#pragma unroll
                for (int x = 0; x < 4; x++)
                {
                    const unsigned px = Byte(w, x);
                    if (!(px & 0x80u)) continue;
                    const float lohi = q ? 0.25f * z[x] + 0.75f * z[x + 1] : 0.75f * z[x] + 0.25f * z[x + 1];
                    ev.v[x] += lohi + (float)(px & 0x3Fu) * (1.0f / 64.0f) * (q ? pC[x + 1] : pC[x]);
                }
                S4(ef + (rI ? o1 : o0), ev);
            }
        }
#pragma unroll
        for (int k = 0; k < 5; k++)
        {
            yM0[k] = yC0[k];
            yM1[k] = yC1[k];
            yC0[k] = yP0[k];
            yC1[k] = yP1[k];
            pC[k] = pP[k];
        }
    }
}

// 3 resident blocks (80 registers, 40 bytes spilled) where the kernel would take 88: measured 14% faster on the 258^3
// level (its grid of one block per SM or so is latency-bound)
__global__ void __launch_bounds__(kPairThreads, 3) k_split_prolong(LevelView fv, LevelView cv,
                                                                const uint8_t *__restrict__ pext,
                                                                const float *__restrict__ ec, float *__restrict__ ef)
{
    PdlWait();
    PdlTrigger();
    SplitProlong(fv, cv, pext, ec, ef, ThisBlk());
}

// The grid of k_split_prolong: threads over (coarse row, fine quad), grid.y chunks of coarse planes sized like
// QuadGrid's (the longest march with a full last wave).
inline dim3 ProlongGridS(const LevelView &fine, const LevelView &coarse, int S)
{
    const long long nq = (long long)(coarse.Nx - 2) * (fine.sRS / 4), perPlane = (nq + kPairThreads - 1) / kPairThreads;
    const long long planes = coarse.Ny - 2 > 0 ? coarse.Ny - 2 : 1;
    return dim3((unsigned)perPlane, (unsigned)((planes + S - 1) / S));
}

inline dim3 ProlongGrid(const LevelView &fine, const LevelView &coarse, int resident)
{
    const long long nq = (long long)(coarse.Nx - 2) * (fine.sRS / 4), perPlane = (nq + kPairThreads - 1) / kPairThreads;
    const long long planes = coarse.Ny - 2 > 0 ? coarse.Ny - 2 : 1;
    const long long bestS = BestMarch(perPlane, planes, (long long)SmCount() * (resident > 0 ? resident : 1));
    return dim3((unsigned)perPlane, (unsigned)((planes + bestS - 1) / bestS));
}

void LaunchSplitProlong(const LevelView &fine, const LevelView &coarse, const uint8_t *pext, const float *eCoarse,
                        float *eFine, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    const int occ = Occ<k_split_prolong>();
    LaunchPdl(k_split_prolong, ProlongGrid(fine, coarse, occ), kPairThreads, 0, st, fine, coarse, pext, eCoarse,
              eFine);
}

// r_c = R res_f = P^T res_f at the coarse unknowns, from the red fine residual. A thread owns four consecutive coarse
// cells K0 .. K0+3 (K0 = 1 + 4 t) of coarse row J (one flat index over (J, t)) and marches along I: fine planes
// 2I-2 .. 2I+1 enter as their (j, k)-weighted 4x4 sums T(a), each kept for the next coarse plane; the red children's
// moved weights enter as X(a). In fine row (a, b) the red cells among k = 2K-2 .. 2K+1 are elements K-1 and K, at
// k = 2K-2+q and 2K+q (q = (a + b) & 1), and the red child of coarse K is element K - q; the five elements
// K0-1 .. K0+3 of a row are one aligned float4 and one more.
__device__ __forceinline__ void SplitRestrictPlane(const LevelView &fv, const uint8_t *__restrict__ pext,
                                                   const float *__restrict__ res, int a, int J, int K0, bool five,
                                                   float T[4], float X[4])
{
#pragma unroll
    for (int x = 0; x < 4; x++) T[x] = X[x] = 0.f;
    if (a > fv.Ny - 1) return;
    const float wt[4] = {0.25f, 0.75f, 0.75f, 0.25f};
#pragma unroll
    for (int dj = 0; dj < 4; dj++)
    {
        const int b = 2 * J - 2 + dj;
        if (b > fv.Nx - 1) continue;
        const int q = (a + b) & 1;
        const long long row = (long long)a * fv.sPS + (long long)b * fv.sRS + (K0 - 1);
        const F4 r4 = L4(res + row);
        const float R[5] = {r4.v[0], r4.v[1], r4.v[2], r4.v[3], five ? res[row + 4] : 0.f};
#pragma unroll
        for (int x = 0; x < 4; x++)
            T[x] += wt[dj] * (q ? 0.75f * R[x] + 0.25f * R[x + 1] : 0.25f * R[x] + 0.75f * R[x + 1]);
        if (dj == 1 || dj == 2)
        {
            const unsigned w = LdU4(pext + row);
            const unsigned w4 = five ? pext[row + 4] : 0u;
#pragma unroll
            for (int x = 0; x < 4; x++)
            {
                // the red child of coarse K0 + x is element K0 + x - q: index x + 1 - q of the five
                const unsigned pw = q ? Byte(w, x) : (x < 3 ? Byte(w, x + 1) : w4);
                X[x] += (float)(pw & 0x3Fu) * R[x + 1 - q];
            }
        }
    }
#pragma unroll
    for (int x = 0; x < 4; x++) X[x] *= 1.0f / 64.0f;
}

__device__ __forceinline__ void SplitRestrictQ(const LevelView &fv, const LevelView &cv,
                                               const uint8_t *__restrict__ pext, const float *__restrict__ res,
                                               float *__restrict__ rc, const Blk &blk)
{
    const int nq = (cv.Nz - 2 + 3) / 4, nt = (cv.Nx - 2) * nq;
    const int t = blk.x * kPairThreads + threadIdx.x;
    if (t >= nt) return;
    const int J = 1 + t / nq, K0 = 1 + 4 * (t - (J - 1) * nq);
    const int S = (cv.Ny - 2 + blk.gy - 1) / blk.gy;
    const int I0 = 1 + blk.y * S, I1 = min(I0 + S, cv.Ny - 1);
    if (I0 >= I1) return;
    const bool five = K0 + 3 <= cv.Nz - 2; // element K0+3 is read only for coarse cell K0+3
    float Tm2[4], Tm1[4], Xm1[4], Xd[4];
    SplitRestrictPlane(fv, pext, res, 2 * I0 - 2, J, K0, five, Tm2, Xd);
    SplitRestrictPlane(fv, pext, res, 2 * I0 - 1, J, K0, five, Tm1, Xm1);
    for (int I = I0; I < I1; I++)
    {
        float T0[4], X0[4], T1[4], X1[4];
        SplitRestrictPlane(fv, pext, res, 2 * I, J, K0, five, T0, X0);
        SplitRestrictPlane(fv, pext, res, 2 * I + 1, J, K0, five, T1, X1);
        const long long c = (long long)I * cv.sI + (long long)J * cv.sJ + K0;
#pragma unroll
        for (int x = 0; x < 4; x++)
        {
            if (K0 + x <= cv.Nz - 2 && (cv.code[c + x] & CODE_UNKNOWN))
                rc[VecIdx(cv, I, J, K0 + x)] =
                    ((0.25f * Tm2[x] + 0.75f * Tm1[x]) + (0.75f * T0[x] + 0.25f * T1[x])) + (Xm1[x] + X0[x]);
            Tm2[x] = T0[x];
            Tm1[x] = T1[x];
            Xm1[x] = X1[x];
        }
    }
}

__global__ void __launch_bounds__(kPairThreads) k_split_restrict(LevelView fv, LevelView cv,
                                                                 const uint8_t *__restrict__ pext,
                                                                 const float *__restrict__ res, float *__restrict__ rc)
{
    PdlWait();
    PdlTrigger();
    SplitRestrictQ(fv, cv, pext, res, rc, ThisBlk());
}

// The same restriction with one thread per coarse cell (K along the 32 lanes, J across the 8 warps), for the smaller
// coarse levels: more threads, and their launches are latency-bound.
__device__ __forceinline__ void SplitRestrictPlane1(const LevelView &fv, const uint8_t *pext, const float *res, int a,
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
        const int q = (a + b) & 1;
        const long long row = (long long)a * fv.sPS + (long long)b * fv.sRS;
        const float lo = res[row + K - 1], hi = res[row + K];
        T += wt[dj] * (q ? 0.75f * lo + 0.25f * hi : 0.25f * lo + 0.75f * hi);
        if (dj == 1 || dj == 2) X += (float)(pext[row + K - q] & 0x3Fu) * (q ? lo : hi);
    }
    X *= 1.0f / 64.0f;
}

// bx, by: the K and J tiles; bz of gz: the chunk of coarse planes
__device__ __forceinline__ void SplitRestrict1(const LevelView &fv, const LevelView &cv,
                                               const uint8_t *__restrict__ pext, const float *__restrict__ res,
                                               float *__restrict__ rc, int bx, int by, int bz, int gz)
{
    const int K = 1 + bx * 32 + threadIdx.x, J = 1 + by * 8 + threadIdx.y;
    if (K > cv.Nz - 2 || J > cv.Nx - 2) return;
    const int S = (cv.Ny - 2 + gz - 1) / gz;
    const int I0 = 1 + bz * S, I1 = min(I0 + S, cv.Ny - 1);
    if (I0 >= I1) return;
    float Tm2, Tm1, Xm1, Xdummy;
    SplitRestrictPlane1(fv, pext, res, 2 * I0 - 2, J, K, Tm2, Xdummy);
    SplitRestrictPlane1(fv, pext, res, 2 * I0 - 1, J, K, Tm1, Xm1);
    for (int I = I0; I < I1; I++)
    {
        float T0, X0, T1, X1;
        SplitRestrictPlane1(fv, pext, res, 2 * I, J, K, T0, X0);
        SplitRestrictPlane1(fv, pext, res, 2 * I + 1, J, K, T1, X1);
        const long long c = (long long)I * cv.sI + (long long)J * cv.sJ + K;
        if (cv.code[c] & CODE_UNKNOWN)
            rc[VecIdx(cv, I, J, K)] = ((0.25f * Tm2 + 0.75f * Tm1) + (0.75f * T0 + 0.25f * T1)) + (Xm1 + X0);
        Tm2 = T0;
        Tm1 = T1;
        Xm1 = X1;
    }
}

__global__ void __launch_bounds__(256) k_split_restrict1(LevelView fv, LevelView cv, const uint8_t *__restrict__ pext,
                                                        const float *__restrict__ res, float *__restrict__ rc)
{
    PdlWait();
    PdlTrigger();
    SplitRestrict1(fv, cv, pext, res, rc, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, (int)gridDim.z);
}

// Coarse levels with at least kRestrictQuadCells cells take the quad kernel (4x fewer loads per coarse cell), the
// smaller ones the per-cell kernel (mode 0); mode 1 takes the per-cell kernel and mode 2 the quad kernel everywhere.
// Both sum the same products in the same order.
constexpr long long kRestrictQuadCells = 1LL << 20;

void LaunchSplitRestrict(const LevelView &fine, const LevelView &coarse, const uint8_t *pext, const float *resFine,
                         float *rCoarse, int mode, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    if (mode == 1 || (mode != 2 && coarse.cells < kRestrictQuadCells))
    {
        const long long perPlane = (long long)((coarse.Nz - 2 + 31) / 32) * ((coarse.Nx - 2 + 7) / 8);
        const int S = MarchPlanes(coarse.Ny - 2, perPlane);
        const dim3 grid((unsigned)((coarse.Nz - 2 + 31) / 32), (unsigned)((coarse.Nx - 2 + 7) / 8),
                        (unsigned)((coarse.Ny - 2 + S - 1) / S));
        LaunchPdl(k_split_restrict1, grid, dim3(32, 8), 0, st, fine, coarse, pext, resFine, rCoarse);
        return;
    }
    const long long nt = (long long)(coarse.Nx - 2) * ((coarse.Nz - 2 + 3) / 4);
    const long long perPlane = (nt + kPairThreads - 1) / kPairThreads, planes = coarse.Ny - 2 > 0 ? coarse.Ny - 2 : 1;
    const long long bestS = BestMarch(perPlane, planes, (long long)SmCount() * Occ<k_split_restrict>());
    LaunchPdl(k_split_restrict, dim3((unsigned)perPlane, (unsigned)((planes + bestS - 1) / bestS)), kPairThreads, 0,
              st, fine, coarse, pext, resFine, rCoarse);
}

// ---------------------------------------------------------------------------------------------------------------
// PCG on a split level 0 (the semantics of k_pair_papply)
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ double SplitRzEff(const double *S, int base, double n, int singular)
{
    return singular ? S[base] - (S[base + 1] / n) * S[base + 2] : S[base];
}

// p_new = U (z - mean + beta p_old), q = M p_new, sum p_new.q, both colours at a thread's quad position.
template <bool kSingular>
__device__ __forceinline__ void SplitPApply(const LevelView &v, const uint8_t *__restrict__ du,
                                            const float *__restrict__ z, float *p0, float *p1, float *__restrict__ q,
                                            const Reducer &R, const double *S, const int *it, int baseEven,
                                            int baseOdd, int slotN, int slotPQ, const Blk &blk)
{
    const int iter = *it, par = iter & 1;
    const float *__restrict__ pIn = par ? p1 : p0;
    float *__restrict__ pOut = par ? p0 : p1;
    const int baseNew = par ? baseOdd : baseEven, baseOld = par ? baseEven : baseOdd;
    const double n = S[slotN];
    const double beta =
        iter == 0 ? 0.0 : SplitRzEff(S, baseNew, n, kSingular) / SplitRzEff(S, baseOld, n, kSingular);
    const float bt = (float)beta;
    const float mean = kSingular ? (float)(S[baseNew + 1] / n) : 0.f;
    const QuadPos P = QuadStart(v, blk);
    if (TileIdle(v, blk.x, P.i0, P.i1))
    {
        double zero[1] = {0.0}; // p and q stay zero on these cells; the block adds its zero term to p.q
        GridReduceB<1>(R, zero, slotPQ, BlkId(blk), BlkCount(blk));
        return;
    }
    const float g = (float)v.gamma, hg = 0.5f * (float)v.gamma;
    const long long hb = v.sHalf;
    auto pn = [&](long long base) {
        const F4 zz = L4(z + base), pv = L4(pIn + base);
        F4 out;
#pragma unroll
        for (int x = 0; x < 4; x++) out.v[x] = (zz.v[x] - mean) + bt * pv.v[x];
        if (kSingular)
        {
            const unsigned d = LdU4(du + base);
#pragma unroll
            for (int x = 0; x < 4; x++) out.v[x] *= Unk(Byte(d, x));
        }
        return out;
    };
    auto pn1 = [&](long long idx) {
        float x = (z[idx] - mean) + bt * pIn[idx];
        if (kSingular) x *= Unk(du[idx]);
        return x;
    };
    const long long b0 = P.off, b1 = hb + P.off;
    F4 M0 = pn(b0 - P.PS), M1 = pn(b1 - P.PS), C0 = pn(b0), C1 = pn(b1);
    float facc = 0.f;
    long long o = 0;
    for (int i = P.i0; i < P.i1; i++, o += P.PS)
    {
        const F4 P0 = pn(b0 + o + P.PS), P1 = pn(b1 + o + P.PS);
        const F4 Jp0 = pn(b0 + o + P.RS), Jp1 = pn(b1 + o + P.RS), Jm0 = pn(b0 + o - P.RS), Jm1 = pn(b1 + o - P.RS);
        const unsigned d0 = LdU4(du + b0 + o), d1 = LdU4(du + b1 + o);
        const int q0 = (i + P.j) & 1, q1 = q0 ^ 1;
        float pw0 = __shfl_up_sync(0xffffffffu, C0.v[3], 1), nx0 = __shfl_down_sync(0xffffffffu, C0.v[0], 1);
        float pw1 = __shfl_up_sync(0xffffffffu, C1.v[3], 1), nx1 = __shfl_down_sync(0xffffffffu, C1.v[0], 1);
        if (P.lane == 0 && P.m0 > 0)
        {
            pw0 = pn1(b0 + o - 1);
            pw1 = pn1(b1 + o - 1);
        }
        if (P.lane == 31 && P.m0 + 4 < P.RS)
        {
            nx0 = pn1(b0 + o + 4);
            nx1 = pn1(b1 + o + 4);
        }
        // colour-0 cells see colour 1 shifted by q0, colour-1 cells see colour 0 shifted by q1
        const F4 sh1 = KShift(C1, pw1, nx1, q0), sh0 = KShift(C0, pw0, nx0, q1);
        F4 Q0, Q1;
#pragma unroll
        for (int x = 0; x < 4; x++)
        {
            const unsigned a0 = Byte(d0, x), a1 = Byte(d1, x);
            const float s0 = ((P1.v[x] + M1.v[x]) + (Jp1.v[x] + Jm1.v[x])) + (C1.v[x] + sh1.v[x]);
            const float s1 = ((P0.v[x] + M0.v[x]) + (Jp0.v[x] + Jm0.v[x])) + (C0.v[x] + sh0.v[x]);
            Q0.v[x] = Unk(a0) * (hg * (float)(a0 & 0x7Fu) * C0.v[x] - g * s0);
            Q1.v[x] = Unk(a1) * (hg * (float)(a1 & 0x7Fu) * C1.v[x] - g * s1);
        }
        if (P.valid)
        {
            S4(pOut + b0 + o, C0);
            S4(pOut + b1 + o, C1);
            S4(q + b0 + o, Q0);
            S4(q + b1 + o, Q1);
#pragma unroll
            for (int x = 0; x < 4; x++) facc += C0.v[x] * Q0.v[x] + C1.v[x] * Q1.v[x];
        }
        M0 = C0;
        M1 = C1;
        C0 = P0;
        C1 = P1;
    }
    double acc[1] = {facc};
    GridReduceB<1>(R, acc, slotPQ, BlkId(blk), BlkCount(blk));
}

template <bool kSingular>
__global__ void __launch_bounds__(kPairThreads, 4)
    k_split_papply(LevelView v, const uint8_t *__restrict__ du, const float *__restrict__ z, float *p0, float *p1,
                   float *__restrict__ q, Reducer R, const double *S, const int *it, int baseEven, int baseOdd,
                   int slotN, int slotPQ)
{
    PdlWait();
    PdlTrigger();
    SplitPApply<kSingular>(v, du, z, p0, p1, q, R, S, it, baseEven, baseOdd, slotN, slotPQ, ThisBlk());
}

void LaunchSplitPApply(const LevelView &v, const uint8_t *du, const float *z, float *p0, float *p1, float *q,
                       const Reducer &R, const double *S, const int *it, int baseEven, int baseOdd, int slotN,
                       int singular, int slotPQ, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    if (singular)
        LaunchPdl(k_split_papply<true>, QuadGrid(v, Occ<k_split_papply<true>>()), kPairThreads, 0, st, v, du, z, p0,
                  p1, q, R, S, it, baseEven, baseOdd, slotN, slotPQ);
    else
        LaunchPdl(k_split_papply<false>, QuadGrid(v, Occ<k_split_papply<false>>()), kPairThreads, 0, st, v, du, z, p0,
                  p1, q, R, S, it, baseEven, baseOdd, slotN, slotPQ);
}

// ---------------------------------------------------------------------------------------------------------------
// the FP64 side of level 0: FP64 arrays in the grid layout, the FP32 vectors colour-split
// ---------------------------------------------------------------------------------------------------------------
// r = sfac * b (split) and (sum b^2, sum b): the residual of a zero iterate. One thread per cell pair (k0 even).
// bx of gx: this block among the launch's blocks (a grid-stride loop)
__device__ __forceinline__ void SplitScaleSum(const LevelView &v, const double *__restrict__ b, float *__restrict__ r,
                                              double sfac, const Reducer &R, int slot, int bx, int gx)
{
    double acc[2] = {0.0, 0.0};
    const long long pairs = v.cells >> 1, stride = (long long)gx * blockDim.x;
    const int H = v.Nz >> 1;
    const double2 *b2 = reinterpret_cast<const double2 *>(b);
    for (long long t = bx * (long long)blockDim.x + threadIdx.x; t < pairs; t += stride)
    {
        const double2 x = b2[t];
        const long long row = t / H; // i * Nx + j
        const int m = (int)(t - row * H);
        const int i = (int)(row / v.Nx), j = (int)(row - (long long)i * v.Nx);
        const int par = (i + j) & 1; // the colour of the pair's first cell
        const long long s = (long long)i * v.sPS + (long long)j * v.sRS + m;
        r[par * v.sHalf + s] = (float)(x.x * sfac);
        r[(par ^ 1) * v.sHalf + s] = (float)(x.y * sfac);
        acc[0] += x.x * x.x + x.y * x.y;
        acc[1] += x.x + x.y;
    }
    GridReduceB<2>(R, acc, slot, (unsigned)bx, (unsigned)gx);
}

constexpr int kScaleSumBlocks = 148 * 8;

__global__ void __launch_bounds__(256) k_split_scale_sum(LevelView v, const double *__restrict__ b,
                                                         float *__restrict__ r, double sfac, Reducer R, int slot)
{
    SplitScaleSum(v, b, r, sfac, R, slot, (int)blockIdx.x, (int)gridDim.x);
}

void LaunchSplitScaleSum(const LevelView &v, const double *b, float *r, double sfac, const Reducer &R, int slot,
                         cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    k_split_scale_sum<<<kScaleSumBlocks, 256, 0, st>>>(v, b, r, sfac, R, slot);
}

// The FP64 refinement step on a uniform split level 0 (k_pair_refine64's, with e read and r written split):
// x_out = x_in + e; r = sfac (b - A x_out) in FP32; (sum (b - A x_out)^2, sum (b - A x_out)) in FP64. One thread per
// cell pair of the grid layout; the pair (k0, k0+1) of row (i, j) is element k0/2 of colours (i+j)&1 and its other.
__device__ __forceinline__ double2 Ld2d(const double *p) { return *reinterpret_cast<const double2 *>(p); }

// 3 resident blocks (80 registers, no spill) beat 4 with a 64-register cap that spills (measured 115 vs 122 us)
__device__ __forceinline__ void SplitRefine64(const LevelView &v, const uint8_t *__restrict__ du,
                                              const double *__restrict__ b, const double *__restrict__ xin,
                                              const float *__restrict__ e, double *__restrict__ xout,
                                              float *__restrict__ r, double scale, double sfac, const Reducer &R,
                                              int slot, const Blk &blk)
{
    const PairPos P = PairStart(v, blk.x, blk.y, blk.gy);
    if (v.act)
    {
        // the block's pairs lie in rows j0 .. j1; with no unknown there, x_out = x_in + e and r stay zero
        const long long c0 = 2LL * kPairThreads * blk.x;
        const int j0 = (int)(c0 / v.Nz), j1 = min(v.Nx - 1, (int)((c0 + 2 * kPairThreads - 1) / v.Nz));
        if (RowsIdle(v, j0, j1, P.i0, P.i1))
        {
            double zero[2] = {0.0, 0.0};
            GridReduceB<2>(R, zero, slot, BlkId(blk), BlkCount(blk));
            return;
        }
    }
    const long long sb = (long long)P.i0 * v.sPS + (long long)P.j * v.sRS + (P.k0 >> 1);
    // the thread's element on plane i0 in colour 0 and colour 1
    const float *e0 = e + sb, *e1 = e + v.sHalf + sb;
    const uint8_t *d0p = du + sb, *d1p = du + v.sHalf + sb;
    float *r0p = r + sb, *r1p = r + v.sHalf + sb;
    const double *xp = xin + P.base;
    // x_in + e at the pair `o` cells (grid layout) / `so` elements (split) away; par: the colour of its first cell
    auto X = [&](long long o, long long so, int par) {
        const double2 a = Ld2d(xp + o);
        const float fa = e0[so], fb = e1[so];
        return make_double2(a.x + (double)(par ? fb : fa), a.y + (double)(par ? fa : fb));
    };
    const int par0 = (P.i0 + P.j) & 1;
    double2 XM = X(-P.sI, -v.sPS, par0 ^ 1), XC = X(0, 0, par0);
    double acc[2] = {0.0, 0.0};
    long long off = 0, so = 0;
    for (int i = P.i0; i < P.i1; i++, off += P.sI, so += v.sPS)
    {
        const int par = (i + P.j) & 1;
        const double2 XP = X(off + P.sI, so + v.sPS, par ^ 1);
        const double2 XJp = X(off + P.sJ, so + v.sRS, par ^ 1), XJm = X(off - P.sJ, so - v.sRS, par ^ 1);
        const double2 bb = Ld2d(b + P.base + off);
        const unsigned da = d0p[so], db = d1p[so];
        const unsigned d0 = par ? db : da, d1 = par ? da : db;
        double left = __shfl_up_sync(0xffffffffu, XC.y, 1);
        double right = __shfl_down_sync(0xffffffffu, XC.x, 1);
        // cell k0-1 is element m-1 of the other colour, cell k0+2 element m+1 of this one (across a row's end: a ring
        // cell's neighbour, masked)
        if (P.lane == 0) left = xp[off - 1] + (double)(par ? e0[so - 1] : e1[so - 1]);
        if (P.lane == 31) right = xp[off + 2] + (double)(par ? e1[so + 1] : e0[so + 1]);
        const double s0 = ((XP.x + XM.x) + (XJp.x + XJm.x)) + (left + XC.y);
        const double s1 = ((XP.y + XM.y) + (XJp.y + XJm.y)) + (XC.x + right);
        const double r0 = (d0 & 0x80u) ? bb.x - scale * (s0 - 0.5 * (double)(d0 & 0x7Fu) * XC.x) : 0.0;
        const double r1 = (d1 & 0x80u) ? bb.y - scale * (s1 - 0.5 * (double)(d1 & 0x7Fu) * XC.y) : 0.0;
        if (P.valid)
        {
            *reinterpret_cast<double2 *>(xout + P.base + off) = XC;
            const float f0 = (float)(r0 * sfac), f1 = (float)(r1 * sfac);
            r0p[so] = par ? f1 : f0;
            r1p[so] = par ? f0 : f1;
            acc[0] += r0 * r0 + r1 * r1;
            acc[1] += r0 + r1;
        }
        XM = XC;
        XC = XP;
    }
    GridReduceB<2>(R, acc, slot, BlkId(blk), BlkCount(blk));
}

// swap (may be null): when *swap is odd, x_in and x_out trade places
__global__ void __launch_bounds__(kPairThreads, 3)
    k_split_refine64(LevelView v, const uint8_t *__restrict__ du, const double *__restrict__ b,
                     const double *xin, const float *__restrict__ e, double *xout,
                     float *__restrict__ r, double scale, double sfac, Reducer R, int slot, const int *swap)
{
    const bool sw = swap && (*swap & 1);
    SplitRefine64(v, du, b, sw ? xout : xin, e, sw ? const_cast<double *>(xin) : xout, r, scale, sfac, R, slot,
                  ThisBlk());
}

void LaunchSplitRefine64(const LevelView &v, const uint8_t *du, const double *b, const double *xin, const float *e,
                         double *xout, float *r, double scale, double sfac, const Reducer &R, int slot,
                         cudaStream_t st, const int *swap)
{
    NB_COUNT_LAUNCH();
    k_split_refine64<<<PairGrid(v, kSplitReduceS), kPairThreads, 0, st>>>(v, du, b, xin, e, xout, r, scale, sfac, R,
                                                                           slot, swap);
}


// ---------------------------------------------------------------------------------------------------------------
// batched launches (nb_batch.cu): grid z = the batch's capacity, block z runs the request at list[z] on the x, y tiles
// of its own grid. The launches that end in a grid-wide sum keep the grid a single solve uses, so each request's sums
// run over its own blocks in the same order whatever else the batch holds; the others take the march length S the
// caller chose (it changes which planes a thread visits, not what a cell gets).
// ---------------------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kPairThreads, 4) kb_split_first(const BatchLevel *__restrict__ lv, int ls, int l,
                                                               BatchList a)
{
    PdlWait();
    PdlTrigger();
    const int q = BatchReqOf(a);
    if (q < 0) return;
    const BatchLevel &L = lv[q * ls + l];
    SplitFirst(L.v, L.du, L.r, L.e, ThisBlk());
}

template <int kDot>
__global__ void __launch_bounds__(kPairThreads, kDot ? 3 : 4)
    kb_split_half(const BatchLevel *__restrict__ lv, int ls, int l, const BatchReq *__restrict__ rq, BatchList a,
                  int colour, int baseEven, int baseOdd, int partSlot)
{
    PdlWait();
    PdlTrigger();
    const int q = BatchReqOf(a);
    if (q < 0) return;
    const BatchLevel &L = lv[q * ls + l];
    const long long h = L.v.sHalf;
    if (kDot)
        SplitHalf<kDot>(L.v, L.du + colour * h, L.r + colour * h, L.e + (colour ^ 1) * h, L.e + colour * h, colour,
                        rq[q].red, rq[q].it, baseEven, baseOdd, partSlot, ThisBlk());
    else
        SplitHalf<kDot>(L.v, L.du + colour * h, L.r + colour * h, L.e + (colour ^ 1) * h, L.e + colour * h, colour,
                        Reducer{}, nullptr, baseEven, baseOdd, partSlot, ThisBlk());
}

__global__ void __launch_bounds__(kPairThreads, 3) kb_split_residual(const BatchLevel *__restrict__ lv, int ls, int l,
                                                                  BatchList a)
{
    PdlWait();
    PdlTrigger();
    const int q = BatchReqOf(a);
    if (q < 0) return;
    const BatchLevel &L = lv[q * ls + l];
    SplitResidual(L.v, L.du, L.r, L.e, L.res, ThisBlk());
}

__global__ void __launch_bounds__(kPairThreads) kb_split_prolong(const BatchLevel *__restrict__ lv, int ls, int l,
                                                                 BatchList a)
{
    PdlWait();
    PdlTrigger();
    const int q = BatchReqOf(a);
    if (q < 0) return;
    const BatchLevel &F = lv[q * ls + l], &C = lv[q * ls + l + 1];
    SplitProlong(F.v, C.v, F.pext, C.e, F.e, ThisBlk());
}

__global__ void __launch_bounds__(kPairThreads) kb_split_restrict(const BatchLevel *__restrict__ lv, int ls, int l,
                                                                  BatchList a)
{
    PdlWait();
    PdlTrigger();
    const int q = BatchReqOf(a);
    if (q < 0) return;
    const BatchLevel &F = lv[q * ls + l], &C = lv[q * ls + l + 1];
    SplitRestrictQ(F.v, C.v, F.pext, F.res, C.r, ThisBlk());
}

// grid (K tiles, J tiles x gz plane chunks, capacity)
__global__ void __launch_bounds__(256) kb_split_restrict1(const BatchLevel *__restrict__ lv, int ls, int l,
                                                         BatchList a, int gyJ, int gz)
{
    PdlWait();
    PdlTrigger();
    const int q = BatchReqOf(a);
    if (q < 0) return;
    const BatchLevel &F = lv[q * ls + l], &C = lv[q * ls + l + 1];
    const int by = (int)blockIdx.y % gyJ, bz = (int)blockIdx.y / gyJ;
    SplitRestrict1(F.v, C.v, F.pext, F.res, C.r, (int)blockIdx.x, by, bz, gz);
}

// form -1: every request in its own form; 0 / 1: only the requests of that form (singular = 1)
__global__ void __launch_bounds__(kPairThreads, 4)
    kb_split_papply(const BatchLevel *__restrict__ lv, int ls, const BatchReq *__restrict__ rq, BatchList a,
                    int baseEven, int baseOdd, int slotN, int slotPQ, int form)
{
    PdlWait();
    PdlTrigger();
    const int q = BatchReqOf(a);
    if (q < 0) return;
    const BatchLevel &L = lv[q * ls];
    const BatchReq &Q = rq[q];
    if (form >= 0 && (Q.singular != 0) != (form == 1)) return;
    if (Q.singular)
        SplitPApply<true>(L.v, L.du, L.e, Q.p0, Q.p1, Q.q, Q.red, Q.red.out, Q.it, baseEven, baseOdd, slotN, slotPQ,
                          ThisBlk());
    else
        SplitPApply<false>(L.v, L.du, L.e, Q.p0, Q.p1, Q.q, Q.red, Q.red.out, Q.it, baseEven, baseOdd, slotN, slotPQ,
                           ThisBlk());
}

__global__ void __launch_bounds__(256) kb_split_scale_sum(const BatchLevel *__restrict__ lv, int ls,
                                                          const BatchReq *__restrict__ rq, BatchList a, int slot)
{
    const int q = BatchReqOf(a);
    if (q < 0) return;
    const BatchLevel &L = lv[q * ls];
    const BatchReq &Q = rq[q];
    SplitScaleSum(L.v, Q.b, L.r, Q.sfac, Q.red, slot, (int)blockIdx.x, (int)gridDim.x);
}

// parity[q]: this pass reads x from xin (0) or xout (1) and writes the other
__global__ void __launch_bounds__(kPairThreads, 3)
    kb_split_refine64(const BatchLevel *__restrict__ lv, int ls, const BatchReq *__restrict__ rq, BatchList a,
                      const int *__restrict__ parity, int slot)
{
    const int q = BatchReqOf(a);
    if (q < 0) return;
    const BatchLevel &L = lv[q * ls];
    const BatchReq &Q = rq[q];
    const bool odd = parity[q] & 1;
    SplitRefine64(L.v, L.du, Q.b, odd ? Q.xout : Q.xin, Q.x, odd ? Q.xin : Q.xout, L.r, Q.scale, Q.sfac, Q.red, slot,
                  ThisBlk());
}

namespace
{
inline dim3 WithZ(dim3 g, int cap)
{
    g.z = (unsigned)cap;
    return g;
}
} // namespace

// the march length a quad kernel's single launch takes on this colour-split level (the default of the batched
// smoothing and residual launches)
int SplitDefaultS(const LevelView &v, int kind)
{
    int occ = 1;
    switch (kind)
    {
    case NB_BK_FIRST: occ = Occ<k_split_first>(); break;
    case NB_BK_HALF: occ = Occ<k_split_half<0>>(); break;
    default: occ = Occ<k_split_residual>(); break;
    }
    const long long planes = v.Ny - 2 > 0 ? v.Ny - 2 : 1;
    const dim3 g = QuadGrid(v, occ);
    return (int)((planes + g.y - 1) / g.y);
}

void LaunchBatchSplit(int kind, const LevelView &v, const LevelView *coarse, int S, int mode,
                      const BatchLevel *lv, int ls, int l, const BatchReq *rq, BatchList a, int cap, int colour,
                      cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    S = S < 1 ? 1 : S;
    switch (kind)
    {
    case NB_BK_FIRST:
        LaunchPdl(kb_split_first, WithZ(QuadGridS(v, S), cap), kPairThreads, 0, st, lv, ls, l, a);
        break;
    case NB_BK_HALF:
        LaunchPdl(kb_split_half<0>, WithZ(QuadGridS(v, S), cap), kPairThreads, 0, st, lv, ls, l, rq, a, colour, 0, 0,
                  0);
        break;
    case NB_BK_RESIDUAL:
        LaunchPdl(kb_split_residual, WithZ(QuadGridS(v, S), cap), kPairThreads, 0, st, lv, ls, l, a);
        break;
    case NB_BK_PROLONG:
        LaunchPdl(kb_split_prolong, WithZ(ProlongGridS(v, *coarse, S), cap), kPairThreads, 0, st, lv, ls, l, a);
        break;
    case NB_BK_RESTRICT:
    {
        const LevelView &c = *coarse;
        const long long planes = c.Ny - 2 > 0 ? c.Ny - 2 : 1;
        const int gz = (int)((planes + S - 1) / S);
        if (mode == 1)
        {
            const int gx = (c.Nz - 2 + 31) / 32, gyJ = (c.Nx - 2 + 7) / 8;
            LaunchPdl(kb_split_restrict1, dim3((unsigned)gx, (unsigned)(gyJ * gz), (unsigned)cap), dim3(32, 8), 0,
                      st, lv, ls, l, a, gyJ, gz);
        }
        else
        {
            const long long nt = (long long)(c.Nx - 2) * ((c.Nz - 2 + 3) / 4);
            const long long perPlane = (nt + kPairThreads - 1) / kPairThreads;
            LaunchPdl(kb_split_restrict, dim3((unsigned)perPlane, (unsigned)gz, (unsigned)cap), kPairThreads, 0, st,
                      lv, ls, l, a);
        }
        break;
    }
    default: break;
    }
}

// The launches that end in a grid-wide sum, on the grids a single solve of the level uses.
void LaunchBatchSplitHalfDot(const LevelView &v, const BatchLevel *lv, int ls, const BatchReq *rq, BatchList a,
                             int cap, int colour, bool last, int baseEven, int baseOdd, int partSlot, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    if (last)
        LaunchPdl(kb_split_half<2>, WithZ(QuadGrid(v, Occ<k_split_half<2>>()), cap), kPairThreads, 0, st, lv, ls, 0,
                  rq, a, colour, baseEven, baseOdd, partSlot);
    else
        LaunchPdl(kb_split_half<1>, WithZ(QuadGrid(v, Occ<k_split_half<1>>()), cap), kPairThreads, 0, st, lv, ls, 0,
                  rq, a, colour, baseEven, baseOdd, partSlot);
}

void LaunchBatchSplitPApply(const LevelView &v, const BatchLevel *lv, int ls, const BatchReq *rq, BatchList a,
                            int cap, int baseEven, int baseOdd, int slotN, int slotPQ, cudaStream_t st)
{
    // a single solve launches its form (singular or not) on that form's grid; both have the same occupancy unless
    // the compiler gave them different register counts, and then each form gets a launch on its own grid
    const dim3 gs = QuadGrid(v, Occ<k_split_papply<true>>()), gn = QuadGrid(v, Occ<k_split_papply<false>>());
    if (gs.x == gn.x && gs.y == gn.y)
    {
        NB_COUNT_LAUNCH();
        LaunchPdl(kb_split_papply, WithZ(gn, cap), kPairThreads, 0, st, lv, ls, rq, a, baseEven, baseOdd, slotN,
                  slotPQ, -1);
        return;
    }
    NB_COUNT_LAUNCHES(2);
    LaunchPdl(kb_split_papply, WithZ(gn, cap), kPairThreads, 0, st, lv, ls, rq, a, baseEven, baseOdd, slotN, slotPQ,
              0);
    LaunchPdl(kb_split_papply, WithZ(gs, cap), kPairThreads, 0, st, lv, ls, rq, a, baseEven, baseOdd, slotN, slotPQ,
              1);
}

void LaunchBatchSplitScaleSum(const BatchLevel *lv, int ls, const BatchReq *rq, BatchList a, int cap, int slot,
                              cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    kb_split_scale_sum<<<dim3(kScaleSumBlocks, 1, cap), 256, 0, st>>>(lv, ls, rq, a, slot);
}

void LaunchBatchSplitRefine64(const LevelView &v, const BatchLevel *lv, int ls, const BatchReq *rq, BatchList a,
                              int cap, const int *parity, int slot, cudaStream_t st)
{
    NB_COUNT_LAUNCH();
    kb_split_refine64<<<WithZ(PairGrid(v, kSplitReduceS), cap), kPairThreads, 0, st>>>(lv, ls, rq, a, parity, slot);
}

// ---------------------------------------------------------------------------------------------------------------
// tile activity: one thread per (plane, tile), ORing the unknown bits of the tile's diagonal bytes in both colours
// ---------------------------------------------------------------------------------------------------------------
constexpr int kTileElems = 4 * kPairThreads;

int SplitActivityTiles(const LevelView &v) { return (v.sPS + kTileElems - 1) / kTileElems; }

__global__ void __launch_bounds__(256) k_split_activity(LevelView v, const uint8_t *__restrict__ du,
                                                        uint8_t *__restrict__ act, int tiles)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)v.Ny * tiles) return;
    const int i = (int)(t / tiles), tile = (int)(t - (long long)i * tiles);
    const int e0 = tile * kTileElems, e1 = min(e0 + kTileElems, v.sPS);
    unsigned any = 0;
    for (int c = 0; c < 2; c++)
    {
        const uint8_t *row = du + (long long)c * v.sHalf + (long long)i * v.sPS;
        for (int e = e0; e < e1; e += 4) any |= LdU4(row + e); // sPS and e0 are multiples of 4
    }
    act[t] = (any & 0x80808080u) ? 1 : 0;
}

void LaunchSplitActivity(const LevelView &v, const uint8_t *du, uint8_t *act, int tiles, cudaStream_t st)
{
    const long long n = (long long)v.Ny * tiles;
    NB_COUNT_LAUNCH();
    k_split_activity<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(v, du, act, tiles);
}

// The occupancy of every split kernel, read outside any stream capture (the launchers size their grids from it).
void PrepareSplitKernels()
{
    (void)Occ<k_split_first>();
    (void)Occ<k_split_half<0>>();
    (void)Occ<k_split_half<1>>();
    (void)Occ<k_split_half<2>>();
    (void)Occ<k_split_residual>();
    (void)Occ<k_split_prolong>();
    (void)Occ<k_split_restrict>();
    (void)Occ<k_split_papply<true>>();
    (void)Occ<k_split_papply<false>>();
}

} // namespace nb
