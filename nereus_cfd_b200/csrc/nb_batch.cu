// Batched solves: many pressure steps of the same grid shape advanced by the same launches (the batched form of the
// mixed-precision solver), and the autotuner of those launches' shapes.
//
// The reference solves one system per call: SolvePressureSystem hands one matrix to Eigen, AMGCL or AMGX and waits
// (src/Methods/PPESolver/PressureSettings.h:578-624). Here a batch holds one solver context per request (its own
// labels, hierarchy, vectors and reductions) and runs the FP32 MG-PCG iterations of all of them together:
//   * every kernel of a CG iteration is ONE launch whose grid z is the batch's capacity; block z serves the request at
//     list[z] of a device-side work list (the requests still iterating), on the x, y tiles of the grid a single
//     solve of that request would use, with that request's level tables (BatchLevel) and scalars (BatchReq);
//   * the iteration is captured once into a CUDA graph whose WHILE node repeats it; after each iteration one block
//     checks every listed request's r.r against its own target and iteration cap, compacts the work list (the
//     converged requests leave it) and ends the loop when the list is empty;
//   * the FP64 refinement around the inner solves is batched the same way, one host synchronisation per pass;
//   * the FP64 steps before and after the solve (ring, right-hand side, compatibility, levelling, scatter,
//     projection) run per request on the batch's stream.
// Each request's sums run over its own blocks in a fixed order, so its result does not depend on the other requests
// of the batch (alone or in any mix, in any slot, the same bits); the autotuner only picks shapes that cannot change
// a result: the march length of the smoothing, residual and transfer kernels, timed on the batch itself and cached
// by (grid, level, kind, capacity). The restriction's kernel (one thread per coarse cell or per four) is not tuned:
// inlined into the batched kernels the two round differently, so it is fixed (per four unless forced). The
// batched kernels inline the same bodies as the single-context ones into other kernels, where the compiler may fuse
// products into FMAs differently, so a batched request and its single-context solve agree to FP32 rounding in the
// inner solve and within the solve's tolerance in the result.
#include "nb_guard.h"

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <sstream>

namespace nb
{

// ---------------------------------------------------------------------------------------------------------------
// the autotuner's cache and choice
// ---------------------------------------------------------------------------------------------------------------
namespace tune
{
struct Choice
{
    int S = 0;    // march length (planes per thread)
    int mode = 0; // restriction: the kernel the level ran (1 per coarse cell, 2 per four); recorded, not chosen
    double us = 0.0;
};
std::mutex g_mu;
std::map<std::string, Choice> g_cache;

static const char *KindName(int kind)
{
    static const char *n[NB_BK_COUNT] = {"first", "half", "residual", "restrict", "prolong"};
    return kind >= 0 && kind < NB_BK_COUNT ? n[kind] : "?";
}

// the cache key: the level's grid (ring included), its depth, the kernel kind and the batch's capacity
std::string Key(int Nx, int Ny, int Nz, int level, int kind, int cap)
{
    char b[96];
    std::snprintf(b, sizeof(b), "split %dx%dx%d L%d %s B%d", Nx, Ny, Nz, level, KindName(kind), cap);
    return b;
}

// The candidate to use given the candidates' measured times: the fastest, unless the fallback (the shape a single
// solve takes) is within 3% of it; among candidates within 0.5% of each other the earlier one. Deterministic in
// its inputs.
int Choose(int n, const double *times, int fallback)
{
    if (n <= 0) return -1;
    int best = -1;
    for (int k = 0; k < n; k++)
    {
        if (!(times[k] > 0.0) || !std::isfinite(times[k])) continue;
        if (best < 0 || times[k] < times[best] * 0.995) best = k;
    }
    if (best < 0) return fallback >= 0 && fallback < n ? fallback : 0;
    if (fallback >= 0 && fallback < n && times[fallback] > 0.0 && times[fallback] <= times[best] * 1.03) return fallback;
    return best;
}

bool Find(const std::string &k, Choice *c)
{
    std::lock_guard<std::mutex> g(g_mu);
    auto it = g_cache.find(k);
    if (it == g_cache.end()) return false;
    *c = it->second;
    return true;
}

void Put(const std::string &k, const Choice &c)
{
    std::lock_guard<std::mutex> g(g_mu);
    g_cache[k] = c;
}

// one line per entry: "<key>|S|mode|us"
std::string Dump()
{
    std::lock_guard<std::mutex> g(g_mu);
    std::ostringstream o;
    for (auto &kv : g_cache)
    {
        char b[64];
        std::snprintf(b, sizeof(b), "|%d|%d|%.3f\n", kv.second.S, kv.second.mode, kv.second.us);
        o << kv.first << b;
    }
    return o.str();
}

// entries of Dump's form; returns the count read, -1 on a malformed line (nothing is then added)
int Load(const char *text)
{
    std::map<std::string, Choice> add;
    std::istringstream in(text ? text : "");
    std::string line;
    while (std::getline(in, line))
    {
        if (line.empty()) continue;
        const size_t a = line.find('|');
        if (a == std::string::npos || a == 0) return -1;
        Choice c;
        if (std::sscanf(line.c_str() + a, "|%d|%d|%lf", &c.S, &c.mode, &c.us) != 3 || c.S < 1 || c.S > 1024 ||
            c.mode < 0 || c.mode > 2)
            return -1;
        add[line.substr(0, a)] = c;
    }
    std::lock_guard<std::mutex> g(g_mu);
    for (auto &kv : add) g_cache[kv.first] = kv.second;
    return (int)add.size();
}

void Clear()
{
    std::lock_guard<std::mutex> g(g_mu);
    g_cache.clear();
}
} // namespace tune

// ---------------------------------------------------------------------------------------------------------------
// small batched kernels: the start of a refinement pass, the inner loop's condition, gathering slots
// ---------------------------------------------------------------------------------------------------------------
// For each request of the pass list: x = 0, p0 = 0 (level 0, colour-split), CG iteration 0, its r.r target and cap;
// the inner work list starts as the pass list.
__global__ void kb_pass_begin(const BatchReq *__restrict__ rq, BatchList pass, int *innerList, int *innerCount,
                              int *loopIters, const double *__restrict__ params)
{
    const int q = BatchReqOf(pass);
    if (q < 0) return;
    const BatchReq Q = rq[q];
    const long long n4 = Q.vecLen >> 2, stride = (long long)gridDim.x * blockDim.x;
    float4 *x4 = reinterpret_cast<float4 *>(Q.x), *p4 = reinterpret_cast<float4 *>(Q.p0);
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n4; t += stride)
    {
        x4[t] = z;
        p4[t] = z;
    }
    for (long long t = 4 * n4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; t < Q.vecLen; t += stride)
    {
        Q.x[t] = 0.f;
        Q.p0[t] = 0.f;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        *Q.it = 0;
        Q.red.out[S_TGT] = params[2 * q];
        Q.red.out[S_MAXIT] = params[2 * q + 1];
        innerList[blockIdx.z] = q;
        if (blockIdx.z == 0)
        {
            *innerCount = *pass.count;
            *loopIters = 0;
        }
    }
}

// After a batched CG iteration: each listed request goes on while its iterations are below its cap and its r.r is
// above its target and finite (the single solve's k_loop_cond); the list keeps those in order, and the WHILE node
// goes on while any is left. The loop also ends after maxLoop iterations whatever the requests' state (every
// request's cap is below it), so it ends by construction. One block of up to 1024 threads (capacity <= 1024).
__global__ void __launch_bounds__(1024) kb_inner_cond(cudaGraphConditionalHandle h, const BatchReq *__restrict__ rq,
                                                      int *list, int *count, int *loopIters, int maxLoop)
{
    __shared__ int warpTot[32];
    const int c = *count, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int q = t < c ? list[t] : -1;
    bool go = false;
    if (q >= 0)
    {
        double *S = rq[q].red.out;
        const int n = *rq[q].it;
        const double rr = S[S_RR];
        S[S_ITS] = (double)n;
        go = n < (int)S[S_MAXIT] && rr > S[S_TGT] && isfinite(rr);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, go);
    if (lane == 0) warpTot[warp] = __popc(bal);
    __syncthreads();
    int before = 0, total = 0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; w++)
    {
        if (w < warp) before += warpTot[w];
        total += warpTot[w];
    }
    before += __popc(bal & ((1u << lane) - 1u));
    __syncthreads(); // every entry is read before any is rewritten
    if (go) list[before] = q;
    if (t == 0)
    {
        const int done = *loopIters + 1;
        *loopIters = done;
        const bool more = total > 0 && done < maxLoop;
        *count = more ? total : 0;
        cudaGraphSetConditional(h, more ? 1u : 0u);
    }
}

// out[q * ns + s] = request q's slot s0 + s, for the listed requests
__global__ void kb_gather(const BatchReq *__restrict__ rq, BatchList a, int s0, int ns, double *out)
{
    const int c = *a.count;
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < c * ns; z += gridDim.x * blockDim.x)
    {
        const int q = a.list[z / ns], s = z % ns;
        out[q * ns + s] = __ldcg(rq[q].red.out + s0 + s);
    }
}

// ---------------------------------------------------------------------------------------------------------------
// the batch
// ---------------------------------------------------------------------------------------------------------------
struct Batch
{
    nb_options opt{};
    int device = 0;
    cudaStream_t st = nullptr;
    bool ownStream = false;
    int cap = 0;
    std::vector<std::unique_ptr<Context>> ctx;

    // device tables: levels [request][ls], requests, the coarse ends' arguments, work lists
    int ls = 0;
    DevArray<BatchLevel> dLev;
    DevArray<BatchReq> dReq;
    DevArray<unsigned char> dTail;
    size_t tailStride = 0, tailSmem = 0;
    DevArray<int> dLists;   // [0, cap): the pass list, [cap, 2 cap): the inner list, [2 cap]: pass count,
                            // [2 cap + 1]: inner count, [2 cap + 2]: the inner loop's iterations
    DevArray<int> dParity;  // per request: this pass's iterate parity
    DevArray<double> dParams, dOut;
    double *hOut = nullptr; // pinned: params (2 cap), gathered slots (4 cap)
    int *hInt = nullptr;    // pinned: the pass list [0, cap), its count [2 cap], the parities [2 cap + 2, 3 cap + 2)
    bool dirty = true;      // a layout changed since the tables were written
    int tableCount = 0;     // the slots the tables hold

    // the shape the graph and the tuning were made for
    std::string shape;
    int nLev = 0, tailStart = 0;
    std::vector<LevelView> views; // slot 0's levels (every request has the same shapes)
    struct LevelTune
    {
        int S[NB_BK_COUNT] = {0, 0, 0, 0, 0};
        int mode = 0;
    };
    std::vector<LevelTune> tuning;
    cudaGraph_t loop = nullptr;
    cudaGraphExec_t loopExec = nullptr;
    long long loopLaunches = 0;
    double tuneMs = 0.0;

    Batch(const nb_options &o, int capacity) : opt(o), cap(capacity)
    {
        device = o.device;
        NB_CK(cudaSetDevice(device));
        if (o.stream)
            st = (cudaStream_t)o.stream;
        else
        {
            NB_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            ownStream = true;
        }
        ctx.resize(cap);
        dLists.alloc(2 * (size_t)cap + 4);
        dLists.zero(st);
        dParity.alloc(cap);
        dParams.alloc(2 * (size_t)cap);
        dOut.alloc(4 * (size_t)cap);
        NB_CK(cudaMallocHost((void **)&hOut, sizeof(double) * 6 * cap));
        NB_CK(cudaMallocHost((void **)&hInt, sizeof(int) * (3 * cap + 2)));
    }

    ~Batch()
    {
        if (st) cudaStreamSynchronize(st);
        ReleaseGraph();
        if (hOut) cudaFreeHost(hOut);
        if (hInt) cudaFreeHost(hInt);
        ctx.clear();
        if (ownStream && st) cudaStreamDestroy(st);
    }

    void ReleaseGraph()
    {
        if (loopExec) cudaGraphExecDestroy(loopExec);
        if (loop) cudaGraphDestroy(loop);
        loopExec = nullptr;
        loop = nullptr;
    }

    BatchList PassList() const { return BatchList{dLists.p, dLists.p + 2 * cap}; }
    BatchList InnerList() const { return BatchList{dLists.p + cap, dLists.p + 2 * cap + 1}; }

    void SetLayout(int slot, int dim, int Nx, int Ny, int Nz, const uint8_t *types, const double *const width[3],
                   const double *const gap[3], int nonUniform, double dh)
    {
        if (slot < 0 || slot >= cap) throw InputError("slot out of range");
        if (!ctx[slot])
        {
            nb_options o = opt;
            o.stream = st;
            o.use_graphs = 0; // the batch captures its own loop; a context's graphs are never built
            ctx[slot].reset(new Context(o));
        }
        ctx[slot]->SetLayout(dim, Nx, Ny, Nz, types, width, gap, nonUniform, dh);
        dirty = true;
    }

    // The batch's shape from slots [0, count): every request a 3D uniform grid of slot 0's sizes whose levels above
    // the coarse end are colour-split (mixed precision); throws InputError otherwise.
    std::string ShapeOf(int count)
    {
        if (count < 1 || count > cap) throw InputError("count out of range");
        for (int i = 0; i < count; i++)
            if (!ctx[i] || !ctx[i]->built) throw InputError("a slot of the batch has no layout");
        Context &A = *ctx[0];
        if (A.opt.precision != NB_PRECISION_MIXED) throw InputError("the batched form runs the mixed precision");
        if (A.dim != 3 || A.nonuniform) throw InputError("the batched form takes uniform 3D grids");
        if (A.tailStart < 1 || A.tailStart >= (int)A.L.size())
            throw InputError("the batched form needs split levels above a shared-memory coarse end");
        for (int l = 0; l < A.tailStart; l++)
            if (!A.Split(l)) throw InputError("the batched form needs colour-split levels above the coarse end");
        for (int i = 1; i < count; i++)
        {
            Context &B = *ctx[i];
            bool same = B.dim == A.dim && B.Nx == A.Nx && B.Ny == A.Ny && B.Nz == A.Nz && !B.nonuniform &&
                        B.L.size() == A.L.size() && B.tailStart == A.tailStart;
            for (size_t l = 0; same && l < A.L.size(); l++)
                same = B.L[l].Nx == A.L[l].Nx && B.L[l].Ny == A.L[l].Ny && B.L[l].Nz == A.L[l].Nz &&
                       B.L[l].sRS == A.L[l].sRS && B.L[l].sHalf == A.L[l].sHalf;
            if (!same) throw InputError("every request of a batch needs the same grid shape");
        }
        char b[128];
        std::snprintf(b, sizeof(b), "%dx%dx%d L%zu T%d pre%d post%d", A.Nx, A.Ny, A.Nz, A.L.size(), A.tailStart,
                      A.PreSweeps(0), A.PostSweeps(0));
        return b;
    }

    void WriteTables(int count)
    {
        Context &A = *ctx[0];
        ls = (int)A.L.size();
        std::vector<BatchLevel> lev((size_t)cap * ls);
        std::vector<BatchReq> req(cap);
        size_t tb = 0, smem = 0;
        {
            std::vector<LevelView> tv;
            for (size_t q = (size_t)A.tailStart; q < A.L.size(); q++) tv.push_back(A.L[q].view());
            TailArgsFor(tv.data(), (int)tv.size(), nullptr, nullptr, 1, 1, 1, nullptr, nullptr, nullptr, &tb, &smem);
        }
        tailStride = (tb + 255) / 256 * 256;
        std::vector<unsigned char> tails(tailStride * cap, 0);
        tailSmem = 0;
        dTail.alloc(tailStride * cap);
        for (int i = 0; i < count; i++)
        {
            Context &C = *ctx[i];
            for (int l = 0; l < ls; l++)
            {
                LevelData &Lv = C.L[l];
                BatchLevel &b = lev[(size_t)i * ls + l];
                b.v = Lv.view();
                b.du = Lv.du.p;
                b.pext = Lv.pext.p;
                b.r = Lv.r32.p;
                b.e = Lv.e32.p;
                b.res = Lv.res32.p;
            }
            BatchReq &r = req[i];
            r.red = C.red;
            r.it = C.iter.p;
            r.singular = C.singular ? 1 : 0;
            r.vecLen = (long long)C.VecLen0();
            r.x = C.x32.p;
            r.p0 = C.p32[0].p;
            r.p1 = C.p32[1].p;
            r.q = C.q32.p;
            r.b = C.b.p;
            r.xin = C.xa.p;
            r.xout = C.xb.p;
            r.scale = C.scale;
            r.sfac = -1.0 / C.scale;
            std::vector<LevelView> tv;
            for (size_t q = (size_t)C.tailStart; q < C.L.size(); q++) tv.push_back(C.L[q].view());
            LevelData &T0 = C.L[C.tailStart];
            size_t bytes = 0, sm = 0;
            TailArgsFor(tv.data(), (int)tv.size(), T0.r32.p, T0.e32.p, C.PreSweeps(C.tailStart),
                        C.PostSweeps(C.tailStart), C.opt.coarse_sweeps, C.tailLists.p, C.tailCounts.p,
                        tails.data() + tailStride * i, &bytes, &sm);
            tailSmem = std::max(tailSmem, sm);
            r.tail = dTail.p + tailStride * i;
        }
        dLev.upload(lev.data(), lev.size(), st);
        dReq.upload(req.data(), req.size(), st);
        NB_CK(cudaMemcpyAsync(dTail.p, tails.data(), tails.size(), cudaMemcpyHostToDevice, st));
        NB_CK(cudaStreamSynchronize(st)); // the host tables above are temporaries
    }

    // the work list [0, count) as the pass list (and the inner count 0)
    void ListAll(int count)
    {
        for (int i = 0; i < count; i++) hInt[i] = i;
        NB_CK(cudaMemcpyAsync(dLists.p, hInt, sizeof(int) * count, cudaMemcpyHostToDevice, st));
        hInt[2 * cap] = count;
        NB_CK(cudaMemcpyAsync(dLists.p + 2 * cap, hInt + 2 * cap, sizeof(int), cudaMemcpyHostToDevice, st));
    }

    // ---- the launches of one batched CG iteration ----
    void Launch(int kind, int l, int colour, BatchList a)
    {
        const LevelTune &T = tuning[l];
        const LevelView *coarse = (kind == NB_BK_RESTRICT || kind == NB_BK_PROLONG) ? &views[l + 1] : nullptr;
        LaunchBatchSplit(kind, views[l], coarse, T.S[kind], T.mode, dLev.p, ls, l, dReq.p, a, cap, colour, st);
    }

    void VCycle(BatchList a)
    {
        Context &A = *ctx[0];
        for (int l = 0; l < tailStart; l++)
        {
            Launch(NB_BK_FIRST, l, 0, a);
            for (int q = 1; q < A.PreSweeps(l); q++)
            {
                Launch(NB_BK_HALF, l, 0, a);
                Launch(NB_BK_HALF, l, 1, a);
            }
            Launch(NB_BK_RESIDUAL, l, 0, a);
            Launch(NB_BK_RESTRICT, l, 0, a);
        }
        LaunchBatchTail(dReq.p, a, cap, tailSmem, st);
        for (int l = tailStart - 1; l >= 0; l--)
        {
            Launch(NB_BK_PROLONG, l, 0, a);
            const int post = A.PostSweeps(l);
            for (int q = 0; q < post; q++)
                for (int c = 1; c >= 0; c--)
                {
                    if (l == 0 && q + 1 == post)
                        LaunchBatchSplitHalfDot(views[0], dLev.p, ls, dReq.p, a, cap, c, c == 0, S_RZ0, S_RZ1, S_RZB,
                                                st);
                    else
                        Launch(NB_BK_HALF, l, c, a);
                }
        }
    }

    void IterBody(BatchList a)
    {
        VCycle(a);
        LaunchBatchSplitPApply(views[0], dLev.p, ls, dReq.p, a, cap, S_RZ0, S_RZ1, S_NUNK, S_PQ, st);
        LaunchBatchLinXR(dLev.p, ls, dReq.p, a, cap, S_RZ0, S_RZ1, S_NUNK, S_PQ, S_RR, st);
    }

    void BuildLoop()
    {
        ReleaseGraph();
        cudaGraphConditionalHandle h = 0;
        NB_CK(cudaGraphCreate(&loop, 0));
        NB_CK(cudaGraphConditionalHandleCreate(&h, loop, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        NB_CK(cudaGraphAddNode(&node, loop, nullptr, 0, &np));
        cudaGraph_t body = np.conditional.phGraph_out[0];
        const long long before = g_launches.load();
        NB_CK(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        const BatchList in = InnerList();
        try
        {
            IterBody(in);
            NB_COUNT_LAUNCH();
            kb_inner_cond<<<1, 1024, 0, st>>>(h, dReq.p, dLists.p + cap, dLists.p + 2 * cap + 1,
                                              dLists.p + 2 * cap + 2, std::max(1, opt.max_iters) + 1);
        }
        catch (...)
        {
            cudaGraph_t dead = nullptr;
            cudaStreamEndCapture(st, &dead);
            ReleaseGraph();
            throw;
        }
        cudaGraph_t out = nullptr;
        NB_CK(cudaStreamEndCapture(st, &out));
        NB_CK(cudaGraphInstantiate(&loopExec, loop, 0));
        loopLaunches = g_launches.load() - before; // counted when run
        NB_COUNT_LAUNCHES(-loopLaunches);
    }

    // ---- the autotuner: per level and kind the march length, on this batch ----
    void Tune(int count)
    {
        tuning.assign(nLev, LevelTune{});
        for (int l = 0; l < tailStart; l++)
        {
            LevelTune &T = tuning[l];
            for (int k = 0; k < NB_BK_COUNT; k++)
                T.S[k] = (k == NB_BK_RESTRICT || k == NB_BK_PROLONG) ? std::min(8, std::max(1, views[l + 1].Ny - 2))
                                                                     : SplitDefaultS(views[l], k);
            // one thread per four coarse cells at every level unless forced: a batched launch has the capacity times
            // a single solve's threads, so the per-cell kernel's extra threads buy nothing (measured on 64 tanks of
            // 128^3: 3.7% faster whole steps than per cell below 2^20 coarse cells, the single solve's rule)
            T.mode = (opt.transfer_kernels == 1 || opt.transfer_kernels == 2) ? opt.transfer_kernels : 2;
        }
        if (!opt.autotune) return;
        cudaEvent_t e0, e1, c0, c1;
        NB_CK(cudaEventCreate(&e0));
        NB_CK(cudaEventCreate(&e1));
        NB_CK(cudaEventCreate(&c0));
        NB_CK(cudaEventCreate(&c1));
        NB_CK(cudaEventRecord(c0, st));
        ListAll(count);
        const BatchList a = PassList();
        auto timeIt = [&](auto &&launch) {
            launch(); // warm
            NB_CK(cudaEventRecord(e0, st));
            for (int r = 0; r < 3; r++) launch();
            NB_CK(cudaEventRecord(e1, st));
            NB_CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            NB_CK(cudaEventElapsedTime(&ms, e0, e1));
            return 1e3 * (double)ms / 3.0;
        };
        for (int l = 0; l < tailStart; l++)
        {
            LevelTune &T = tuning[l];
            for (int k = 0; k < NB_BK_COUNT; k++)
            {
                const LevelView &plane = (k == NB_BK_RESTRICT || k == NB_BK_PROLONG) ? views[l + 1] : views[l];
                const int planes = std::max(1, plane.Ny - 2);
                const LevelView &v = views[l];
                const std::string key = tune::Key(v.Nx, v.Ny, v.Nz, l, k, cap);
                tune::Choice c;
                // a cached entry gives the march only: the restriction's kernel stays the fixed rule's, whatever an
                // entry records, since the two kernels do not give the same bits in the batched form
                if (tune::Find(key, &c))
                {
                    T.S[k] = c.S;
                    continue;
                }
                // candidates: the default march first, then marches of 1 .. 32 planes
                const int mode = k == NB_BK_RESTRICT ? T.mode : 0;
                std::vector<int> cands{T.S[k]};
                for (int S = 1; S <= 32; S *= 2)
                {
                    if (S > planes && S != 1) break;
                    if (S != cands[0]) cands.push_back(S);
                }
                std::vector<double> times;
                for (const int S : cands)
                    times.push_back(timeIt([&] {
                        const LevelView *coarse = (k == NB_BK_RESTRICT || k == NB_BK_PROLONG) ? &views[l + 1] : nullptr;
                        LaunchBatchSplit(k, views[l], coarse, S, mode, dLev.p, ls, l, dReq.p, a, cap, 0, st);
                    }));
                const int pick = tune::Choose((int)times.size(), times.data(), 0);
                c.S = cands[pick];
                c.mode = mode;
                c.us = times[pick];
                tune::Put(key, c);
                T.S[k] = c.S;
            }
        }
        NB_CK(cudaEventRecord(c1, st));
        NB_CK(cudaEventSynchronize(c1));
        float ms = 0.f;
        NB_CK(cudaEventElapsedTime(&ms, c0, c1));
        tuneMs += ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(c0);
        cudaEventDestroy(c1);
        // the timed launches wrote the levels' e, res and the coarse r; each is rewritten before it is read in a
        // solve (the first sweep writes e, the residual res, the restriction r), and they kept zero off the unknowns
    }

    // ---- one batched pressure step of requests [0, count) ----
    int Project(int count, const nb_batch_item *items, nb_result *res)
    {
        for (int i = 0; i < count; i++)
            if (!(items[i].tol > 0.0)) throw InputError("tolerance must be positive");
        const std::string sh = ShapeOf(count);
        Context &A = *ctx[0];
        if (sh != shape)
        {
            shape = sh;
            nLev = (int)A.L.size();
            tailStart = A.tailStart;
            views.clear();
            for (auto &Lv : A.L) views.push_back(Lv.view());
            PrepareSplitKernels();
            PrepareTail<float>(kTailMaxSmem);
            dirty = true;
            tuning.clear();
            ReleaseGraph();
        }
        if (dirty || count > tableCount)
        {
            WriteTables(count);
            dirty = false;
            tableCount = count;
        }
        if (tuning.size() != (size_t)nLev)
        {
            Tune(count);
            ReleaseGraph();
        }
        if (!loopExec) BuildLoop();

        cudaEvent_t ev0, ev1;
        NB_CK(cudaEventCreate(&ev0));
        NB_CK(cudaEventCreate(&ev1));
        NB_CK(cudaEventRecord(ev0, st));
        // ring, right-hand side, compatibility per request
        for (int i = 0; i < count; i++)
        {
            const nb_batch_item &it = items[i];
            ctx[i]->BatchBegin(it.u, it.v, it.w, it.p, it.rho, it.dt, it.needs_compat);
            ctx[i]->xa.zero(st);
        }
        // the residual of x = 0 and ||b||^2 for all
        ListAll(count);
        LaunchBatchSplitScaleSum(dLev.p, ls, dReq.p, PassList(), cap, S_RES, st);
        NB_COUNT_LAUNCH();
        kb_gather<<<1, 256, 0, st>>>(dReq.p, PassList(), S_RES, 2, dOut.p);
        NB_CK(cudaMemcpyAsync(hOut, dOut.p, sizeof(double) * 2 * count, cudaMemcpyDeviceToHost, st));
        NB_CK(cudaStreamSynchronize(st));
        struct State
        {
            double bn2, rr64, tolEff;
            int outer, inner, status, parity;
        };
        std::vector<State> S(count);
        for (int i = 0; i < count; i++)
        {
            S[i] = State{hOut[2 * i], hOut[2 * i], items[i].tol, 0, 0, NB_OK, 0};
            if (ctx[i]->n == 0) S[i].bn2 = S[i].rr64 = 0.0;
        }
        const int maxOuter = std::max(1, opt.max_outer);
        long long passes = 0;
        while (true)
        {
            int np = 0;
            for (int i = 0; i < count; i++)
            {
                State &s = S[i];
                if (!(s.bn2 > 0.0)) continue;
                if (std::sqrt(s.rr64 / s.bn2) <= s.tolEff || s.status != NB_OK) continue;
                if (s.outer >= maxOuter || !std::isfinite(s.rr64))
                {
                    s.status = NB_NOT_CONVERGED;
                    continue;
                }
                const double sf = -1.0 / ctx[i]->scale, rr0 = s.rr64 * sf * sf;
                hInt[np++] = i;
                hOut[2 * i] = Context::InnerTarget(rr0, ctx[i]->InnerTol(s.tolEff), s.tolEff, s.bn2, sf);
                hOut[2 * i + 1] = (double)std::max(1, opt.max_iters);
                hInt[2 * cap + 2 + i] = s.parity;
            }
            if (np == 0) break;
            hInt[2 * cap] = np;
            NB_CK(cudaMemcpyAsync(dLists.p, hInt, sizeof(int) * np, cudaMemcpyHostToDevice, st));
            NB_CK(cudaMemcpyAsync(dLists.p + 2 * cap, hInt + 2 * cap, sizeof(int), cudaMemcpyHostToDevice, st));
            NB_CK(cudaMemcpyAsync(dParams.p, hOut, sizeof(double) * 2 * count, cudaMemcpyHostToDevice, st));
            NB_CK(cudaMemcpyAsync(dParity.p, hInt + 2 * cap + 2, sizeof(int) * count, cudaMemcpyHostToDevice, st));
            NB_COUNT_LAUNCH();
            kb_pass_begin<<<dim3(64, 1, cap), 256, 0, st>>>(dReq.p, PassList(), dLists.p + cap,
                                                            dLists.p + 2 * cap + 1, dLists.p + 2 * cap + 2,
                                                            dParams.p);
            NB_CK(cudaGraphLaunch(loopExec, st));
            LaunchBatchSplitRefine64(views[0], dLev.p, ls, dReq.p, PassList(), cap, dParity.p, S_RES, st);
            NB_COUNT_LAUNCH();
            kb_gather<<<1, 256, 0, st>>>(dReq.p, PassList(), S_RES, 2, dOut.p);
            NB_COUNT_LAUNCH();
            kb_gather<<<1, 256, 0, st>>>(dReq.p, PassList(), S_ITS, 1, dOut.p + 2 * cap);
            NB_CK(cudaMemcpyAsync(hOut + 2 * cap, dOut.p, sizeof(double) * 3 * cap, cudaMemcpyDeviceToHost, st));
            NB_CK(cudaStreamSynchronize(st));
            NB_CK(cudaGetLastError());
            int maxIts = 0;
            for (int z = 0; z < np; z++)
            {
                const int i = hInt[z];
                State &s = S[i];
                const int n = (int)hOut[4 * cap + i];
                s.inner += n;
                maxIts = std::max(maxIts, n);
                s.rr64 = hOut[2 * cap + 2 * i];
                s.parity ^= 1;
                s.outer++;
            }
            NB_COUNT_LAUNCHES(maxIts * loopLaunches); // the loop ran as many iterations as its longest request
            passes++;
        }
        // levelling, scatter, ring, velocity correction per request; max |div u| for all
        for (int i = 0; i < count; i++)
        {
            Context &C = *ctx[i];
            double *x = S[i].parity ? C.xb.p : C.xa.p;
            const nb_batch_item &it = items[i];
            C.BatchEnd(x, it.u, it.v, it.w, it.p, it.rho, it.dt, it.needs_compat);
        }
        ListAll(count);
        NB_COUNT_LAUNCH();
        kb_gather<<<1, 256, 0, st>>>(dReq.p, PassList(), S_DIV, 1, dOut.p);
        NB_CK(cudaMemcpyAsync(hOut, dOut.p, sizeof(double) * count, cudaMemcpyDeviceToHost, st));
        NB_CK(cudaEventRecord(ev1, st));
        NB_CK(cudaEventSynchronize(ev1));
        NB_CK(cudaGetLastError());
        float ms = 0.f;
        NB_CK(cudaEventElapsedTime(&ms, ev0, ev1));
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        int worst = NB_OK;
        for (int i = 0; i < count; i++)
        {
            nb_result &r = res[i];
            std::memset(&r, 0, sizeof(r));
            Context &C = *ctx[i];
            r.n = C.n;
            r.singular = C.singular ? 1 : 0;
            r.levels = (int)C.L.size();
            r.iters_outer = S[i].outer;
            r.iters_inner = S[i].inner;
            r.b_norm = std::sqrt(S[i].bn2);
            r.rel_res = S[i].bn2 > 0.0 ? std::sqrt(S[i].rr64 / S[i].bn2) : 0.0;
            r.max_div = hOut[i];
            r.seconds = ms * 1e-3;
            r.status = S[i].status;
            C.lastIterations = r.iters_inner;
            if (r.status != NB_OK) worst = r.status;
        }
        return worst;
    }
};

} // namespace nb

struct nb_batch
{
    std::unique_ptr<nb::Batch> b;
};

using nb::capi::Fail;
using nb::capi::Guard;

extern "C" {

int nereus_b200_batch_create(nb_batch **batch, const nb_options *opt, int capacity)
{
    if (!batch) return Fail(NB_BAD_INPUT, "batch is null");
    *batch = nullptr;
    if (capacity < 1 || capacity > 1024) return Fail(NB_BAD_INPUT, "capacity must be 1 .. 1024");
    return Guard([&] {
        nb_options o;
        nereus_b200_default_options(&o);
        if (opt) o = *opt;
        if (o.precision != NB_PRECISION_MIXED) throw nb::InputError("the batched form runs the mixed precision");
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return Fail(NB_NO_DEVICE, "no CUDA device");
        if (o.device < 0 || o.device >= count) throw nb::InputError("device ordinal out of range");
        auto *h = new nb_batch;
        try
        {
            h->b.reset(new nb::Batch(o, capacity));
        }
        catch (...)
        {
            delete h;
            throw;
        }
        *batch = h;
        return (int)NB_OK;
    });
}

void nereus_b200_batch_destroy(nb_batch *batch)
{
    if (!batch) return;
    try
    {
        if (batch->b) cudaSetDevice(batch->b->device);
        batch->b.reset();
    }
    catch (...)
    {
    }
    delete batch;
}

int nereus_b200_batch_set_layout(nb_batch *batch, int slot, int dim, int Nx, int Ny, int Nz, const uint8_t *cellTypes,
                                 const double *const width[3], const double *const gap[3], int nonUniform, double dh)
{
    if (!batch || !batch->b) return Fail(NB_BAD_INPUT, "batch is null");
    return Guard([&] {
        NB_CK(cudaSetDevice(batch->b->device));
        batch->b->SetLayout(slot, dim, Nx, Ny, Nz, cellTypes, width, gap, nonUniform, dh);
        return (int)NB_OK;
    });
}

int nereus_b200_batch_project_device(nb_batch *batch, int count, const nb_batch_item *items, nb_result *results)
{
    if (!batch || !batch->b) return Fail(NB_BAD_INPUT, "batch is null");
    if (!items || !results) return Fail(NB_BAD_INPUT, "null items or results");
    return Guard([&] {
        NB_CK(cudaSetDevice(batch->b->device));
        return batch->b->Project(count, items, results);
    });
}

int nereus_b200_batch_info(nb_batch *batch, nb_batch_info *info)
{
    if (!batch || !batch->b || !info) return Fail(NB_BAD_INPUT, "null argument");
    const nb::Batch &B = *batch->b;
    std::memset(info, 0, sizeof(*info));
    info->capacity = B.cap;
    info->levels = B.nLev;
    info->tail_start = B.tailStart;
    info->loop_launches = B.loopLaunches;
    info->tune_ms = B.tuneMs;
    for (int l = 0; l < B.tailStart && l < NB_BATCH_MAX_LEVELS; l++)
    {
        for (int k = 0; k < nb::NB_BK_COUNT; k++) info->march[l][k] = B.tuning[l].S[k];
        info->restrict_mode[l] = B.tuning[l].mode;
    }
    return NB_OK;
}

int nereus_b200_tune_choose(int n, const double *times, int fallback)
{
    if (n < 1 || !times) return Fail(NB_BAD_INPUT, "no candidates");
    return nb::tune::Choose(n, times, fallback);
}

int nereus_b200_tune_key(int Nx, int Ny, int Nz, int level, int kind, int capacity, char *buf, int size)
{
    if (!buf || size < 1) return Fail(NB_BAD_INPUT, "null buffer");
    if (kind < 0 || kind >= nb::NB_BK_COUNT) return Fail(NB_BAD_INPUT, "unknown kernel kind");
    const std::string k = nb::tune::Key(Nx, Ny, Nz, level, kind, capacity);
    std::snprintf(buf, (size_t)size, "%s", k.c_str());
    return (int)k.size();
}

int nereus_b200_tune_cache_dump(char *buf, int size)
{
    const std::string t = nb::tune::Dump();
    if (buf && size > 0) std::snprintf(buf, (size_t)size, "%s", t.c_str());
    return (int)t.size();
}

int nereus_b200_tune_cache_load(const char *text)
{
    const int n = nb::tune::Load(text);
    if (n < 0) return Fail(NB_BAD_INPUT, "malformed tuning cache text");
    return n;
}

void nereus_b200_tune_cache_clear(void) { nb::tune::Clear(); }

} // extern "C"
