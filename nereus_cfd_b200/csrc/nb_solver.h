// Host orchestration of the B200 pressure projection: the multigrid hierarchy, the PCG and refinement drivers, the
// projection pipeline. One Context serves one grid on one device and stream.
#pragma once

#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "nb_kernels.h"

namespace nb
{

struct CudaError : std::runtime_error
{
    cudaError_t code;
    CudaError(const char *what, cudaError_t c)
        : std::runtime_error(std::string(what) + ": " + cudaGetErrorString(c)), code(c) {}
};

struct InputError : std::runtime_error
{
    explicit InputError(const std::string &s) : std::runtime_error(s) {}
};

#define NB_CK(x)                                                                                                   \
    do                                                                                                             \
    {                                                                                                              \
        cudaError_t e_ = (x);                                                                                      \
        if (e_ != cudaSuccess) throw ::nb::CudaError(#x, e_);                                                      \
    } while (0)

// The device memory a context's layout-dependent arrays live in: a stream-ordered pool of the context's own
// (cudaMemPool, nothing released back until the context goes), allocated from and freed to on the context's stream,
// so the work that used memory is ordered before its next use. A layout change reuses what the context already holds,
// suballocated by the driver for any size. Plain allocation was measured stalling a busy server: with 4 slots each
// changing shape per request, cudaMalloc took 10-66 ms even for a few hundred bytes, and every request in flight
// waited with it (up to 300 ms); cudaFree waits for the whole device.
struct ArrayPool
{
    cudaMemPool_t pool = nullptr;
    cudaStream_t st = nullptr; // allocations and frees are ordered on it (null: the legacy stream)
    ArrayPool() = default;
    ArrayPool(const ArrayPool &) = delete;
    ArrayPool &operator=(const ArrayPool &) = delete;
    ~ArrayPool()
    {
        if (pool) cudaMemPoolDestroy(pool); // its memory is released once every allocation from it is freed
    }
    void Init(int device, cudaStream_t s)
    {
        cudaMemPoolProps pr = {};
        pr.allocType = cudaMemAllocationTypePinned;
        pr.location.type = cudaMemLocationTypeDevice;
        pr.location.id = device;
        NB_CK(cudaMemPoolCreate(&pool, &pr));
        unsigned long long keep = ~0ull; // the attribute is a 64-bit unsigned
        NB_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        st = s;
    }
    // null when the stream is being captured (the caller allocates plainly then)
    void *Get(size_t bytes)
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (!pool || cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return nullptr;
        void *p = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, st);
        if (e == cudaErrorMemoryAllocation)
        {
            // memory the pool keeps but nothing uses goes back to the device, then once more
            cudaGetLastError();
            cudaStreamSynchronize(st);
            cudaMemPoolTrimTo(pool, 0);
            e = cudaMallocFromPoolAsync(&p, bytes, pool, st);
        }
        if (e != cudaSuccess) throw CudaError("cudaMallocFromPoolAsync", e);
        // zeroed: a batched solve was measured to differ with the memory's earlier contents once it was recycled
        // (some cells are read that no kernel of the layout writes), as it never did from fresh cudaMalloc memory
        NB_CK(cudaMemsetAsync(p, 0, bytes, st));
        return p;
    }
    void Put(void *p) { cudaFreeAsync(p, st); }
};

// the pool that DevArray allocations made on this thread draw on (set by a Context around its layout work)
inline thread_local ArrayPool *t_arrayPool = nullptr;
struct ArrayPoolScope
{
    ArrayPool *prev;
    explicit ArrayPoolScope(ArrayPool *c) : prev(t_arrayPool) { t_arrayPool = c; }
    ~ArrayPoolScope() { t_arrayPool = prev; }
};

// A device array that keeps its allocation: a smaller or equal size reuses it (no cudaFree, which would synchronize
// the device, and no cudaMalloc), a larger one replaces it. Allocated under an ArrayPoolScope, it takes its memory
// from that pool and gives it back there.
template <typename T> struct DevArray
{
    T *p = nullptr;
    size_t n = 0, cap = 0;
    ArrayPool *pool = nullptr; // where p came from (null: cudaMalloc)
    DevArray() = default;
    DevArray(const DevArray &) = delete;
    DevArray &operator=(const DevArray &) = delete;
    DevArray(DevArray &&o) noexcept : p(o.p), n(o.n), cap(o.cap), pool(o.pool)
    {
        o.p = nullptr;
        o.n = o.cap = 0;
        o.pool = nullptr;
    }
    DevArray &operator=(DevArray &&o) noexcept
    {
        if (this != &o)
        {
            release();
            p = o.p; n = o.n; cap = o.cap; pool = o.pool;
            o.p = nullptr; o.n = o.cap = 0; o.pool = nullptr;
        }
        return *this;
    }
    ~DevArray() { release(); }
    void alloc(size_t count)
    {
        if (count == 0) { n = 0; return; }
        if (p && count <= cap) { n = count; return; }
        ArrayPool *c = t_arrayPool ? t_arrayPool : pool;
        release();
        if (c && (p = (T *)c->Get(count * sizeof(T))) != nullptr)
        {
            pool = c;
            n = cap = count;
            return;
        }
        pool = nullptr;
        cudaError_t e = cudaMalloc((void **)&p, count * sizeof(T));
        if (e != cudaSuccess) { p = nullptr; throw CudaError("cudaMalloc", e); }
        n = cap = count;
    }
    void zero(cudaStream_t st) { if (p && n) NB_CK(cudaMemsetAsync(p, 0, n * sizeof(T), st)); }
    void upload(const T *h, size_t count, cudaStream_t st)
    {
        alloc(count);
        if (count) NB_CK(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
    }
    void release()
    {
        if (p)
        {
            if (pool) pool->Put(p);
            else cudaFree(p);
        }
        p = nullptr;
        n = cap = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// scalar slots of the reducer
enum : int
{
    S_RZ0 = 0,   // (r.z, sum z, sum r), even iterations
    S_RZ1 = 3,   // ... odd iterations
    S_PQ = 6,
    S_RR = 7,
    S_RES = 8,   // ||b - A x||^2, sum (b - A x)
    S_SUM = 10,  // compensated sum (sum, carry)
    S_DIV = 12,
    S_NUNK = 14, // the count of unknowns, read by the CG kernels on the device
    S_RZB = 16,  // (r.z, sum z, sum r) of the black cells, summed by the black half of the last sweep
    S_TGT = 19,  // the device-side CG loop: r.r target, iteration cap, iterations done
    S_MAXIT = 20,
    S_ITS = 21,
    S_BN2 = 22,  // the device-side refinement loop: ||b||^2, the tolerance, the CG iterations of all passes
    S_TOL = 23,
    S_INNER = 24,
    S_INTOL = 25, // the inner solves' relative tolerance of this solve (InnerTol)
    S_COUNT = 26
};

struct LevelData
{
    int dim = 3, Nx = 0, Ny = 0, Nz = 1;
    long long cells = 0;
    bool stretched = false;
    double gamma = 1.0;
    std::vector<double> w[3], g[3];
    // the device copies of w, g (FP64) and of w, 1/g (FP32): pointers into the context's packed table array
    const double *dw[3] = {}, *dg[3] = {};
    const float *dw32[3] = {}, *dig32[3] = {};
    // the x groups of the transfer to the next coarser level (LevelView::xp, xr) and their device copies in the
    // packed table array; empty: x cells paired by two like the other axes
    std::vector<int> xp, xr;
    const int *dxp = nullptr, *dxr = nullptr;
    DevArray<uint8_t> types, code;
    DevArray<uint8_t> du;                 // diagonal units for the pair kernels (nb_pairs.cu); empty elsewhere.
                                          // Colour-split level: in that layout, and the codes on a stretched level
    DevArray<uint8_t> pext;               // unknown flag + moved prolongation weight toward the next coarser level
                                          // (colour-split level: the red cells only)
    DevArray<uint8_t> act;                // colour-split level: which (plane, tile) holds an unknown (LevelView::act)
    int actTiles = 0;
    // the colour-split layout of the FP32 vectors (nb_split.cu); sRS = 0: the grid layout
    int sRS = 0, sPS = 0;
    long long sHalf = 0;
    size_t VecLen() const { return sRS ? (size_t)(2 * sHalf) : (size_t)cells; }
    DevArray<float> r32, e32, res32;
    DevArray<double> r64, e64, res64;
    LevelView view() const;
    template <typename T> T *r();
    template <typename T> T *e();
    template <typename T> T *res();
};

struct Context
{
    ArrayPool arrays; // first, so that it outlives every array that gives its memory back to it
    nb_options opt{};
    int device = 0;
    cudaStream_t st = nullptr;
    bool ownStream = false;

    // layout
    bool built = false;
    int dim = 3, Nx = 0, Ny = 0, Nz = 1;
    bool nonuniform = false;
    double dh = 1.0, scale = 1.0;
    std::vector<uint8_t> layout;
    std::vector<double> wt[3], gt[3];
    std::vector<LevelData> L;
    int tailStart = 0;                       // levels from here down run in one shared-memory block (nb_tail.cu)
    DevArray<uint8_t> tables;                // every level's spacing tables, packed (UploadTables)
    uint8_t *tablesHost = nullptr;           // their pinned staging buffer
    size_t tablesHostCap = 0;
    DevArray<unsigned> tailLists;            // the tail levels' per-colour lists of unknowns (built per layout)
    DevArray<int> tailCounts;
    DevArray<int32_t> idp;
    bool idpValid = false; // the numbering is made when first asked for (GetIdp, ExportMatrix, SolveLaplacian, Rhs)
    int n = 0;
    bool singular = false;
    DevArray<int> lineCounts, lineOffsets;
    DevArray<uint8_t> scanTmp;
    size_t scanTmpBytes = 0;

    // solver vectors on level 0 (grid layout)
    DevArray<double> b, xa, xb;
    DevArray<float> p32[2], q32, x32;
    DevArray<double> p64[2], q64;

    // fields for the host-buffer entry points
    DevArray<double> du, dv, dw, dp, dpPrev;
    DevArray<double> pSave, dq; // the incremental scheme's prescribed ring values and known Dirichlet increments

    // reductions
    DevArray<double> partials, slots;
    DevArray<unsigned> counter;
    double *hostSlots = nullptr; // pinned
    Reducer red{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // host-buffer projection (nereus_b200_project): when hostP is set, ProjectDevice copies the final p there on the
    // copy stream cst as soon as it is final, beside the velocity correction, then u, v, w to hostU, hostV, hostW as
    // soon as they are corrected, beside the divergence check, and sets hostCopied; evPDone marks the copies' end
    double *hostP = nullptr, *hostU = nullptr, *hostV = nullptr, *hostW = nullptr;
    bool hostCopied = false;
    cudaStream_t cst = nullptr;
    cudaEvent_t evP = nullptr, evPDone = nullptr;

    int lastIterations = 0;

    // per-kernel device timing (nereus_b200_profile_*): CUDA events around the selected launches, on the context's
    // stream, or as event nodes inside a captured iteration graph, summed per kernel id
    struct ProfRecord
    {
        int id;
        cudaEvent_t a, b;
        double bytes;      // of all the launches between the two events
        int launches = 1;  // launches of kernel `id` between them (back to back)
    };
    struct ProfTotal
    {
        long long launches = 0;
        double ms = 0.0, bytes = 0.0;
    };
    unsigned profMask = 0;
    std::vector<cudaEvent_t> evPool;
    size_t evUsed = 0;
    std::vector<ProfRecord> prof;    // stream launches not yet read
    ProfTotal profTot[NB_K_COUNT];
    int profOpen = -1;
    cudaEvent_t profA = nullptr;
    double profBytes = 0.0;
    int profLaunches = 1;
    // events around the next `launches` launches of kernel `id` (back to back on the stream), `bytes` in all
    void ProfBegin(int id, double bytes, int launches = 1);
    void ProfEnd(int launches = -1); // launches >= 0: the bracket's kernel count, set at its end
    bool profQuiet = false;          // inside a bracket that covers several kernels: their own brackets are skipped
    template <typename T> void CoarseBracket(int l, T *r, T *e);
    void ProfClear();
    void ProfFlush();
    void ProfRead(int id, int *launches, double *ms, double *bytesPerLaunch);

    // one captured CG iteration (V-cycle, r.z, direction update + apply, x/r update, rr to the host) per precision
    struct IterGraph
    {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t exec = nullptr;
        std::vector<ProfRecord> prof;
        std::vector<cudaEvent_t> events;
        unsigned mask = 0;
        long long launches = 0; // kernels one replay runs
        // the whole CG loop as one graph: a WHILE node whose body is the iteration, the condition set on the device
        // (no profiling events inside); built once, or marked unavailable when the runtime refuses it
        cudaGraph_t loop = nullptr;
        cudaGraphExec_t loopExec = nullptr;
        long long loopLaunches = 0; // kernels one loop iteration runs
        bool loopFailed = false;
        void Release();
    };
    IterGraph graphs[2]; // [0] float, [1] double
    IterGraph *capturing = nullptr;
    DevArray<int> iter;  // the CG iteration number, advanced on the device
    // the whole mixed solve as one graph: the zero-iterate residual, then a WHILE node over refinement passes whose
    // body holds the CG loop's WHILE node and the FP64 refinement step (built once per shape, or unavailable)
    cudaGraph_t solveGraph = nullptr;
    cudaGraphExec_t solveExec = nullptr;
    bool solveFailed = false;
    long long solvePrologLaunches = 0, solvePassLaunches = 0, solveIterLaunches = 0;
    DevArray<int> passes; // the refinement passes done (their parity picks the iterate the next pass reads)
    void ReleaseSolveGraph();

    Context(const nb_options &o);
    ~Context();

    void SetLayout(int dim, int Nx, int Ny, int Nz, const uint8_t *types, const double *const width[3],
                   const double *const gap[3], int nonUniform, double dh);
    // The pressure step and projection on device fields; returns the nb_status.
    // solve: the pressure step (ring, RHS, compatibility, solve, level, scatter, ring); correct: the velocity
    // correction with the p that results.
    // pPrev: p^n with its ring (the reference's gridAnt->p), used by the incremental scheme (required) and by the
    // Chorin warm start (warm = true; uniform grids only, as WarmStartEnabled, PressureSolver3D.cpp:215-220).
    int ProjectDevice(double *u, double *v, double *w, double *p, double rho, double dt, int compat, double tol,
                      nb_result *out, bool solve = true, bool correct = true, const double *pPrev = nullptr,
                      int scheme = NB_SCHEME_CHORIN, bool warm = false);
    int SolveLaplacian(const double *f, double *x, double tol, nb_result *out);
    // A batch's halves of the Chorin step around its solve (nb_batch.cu), on this context's stream: Begin checks the
    // call and runs the ring, the right-hand side and the compatibility step; End levels x, scatters it into p, runs
    // the ring and the velocity correction and leaves max |div u| in slot S_DIV.
    void BatchBegin(double *u, double *v, double *w, double *p, double rho, double dt, int compat);
    void BatchEnd(double *x, double *u, double *v, double *w, double *p, double rho, double dt, int compat);
    void Rhs(const double *u, const double *v, const double *w, const double *p, double rho, double dt, double *bOut);
    void ExportMatrix(int32_t *rowptr, int32_t *col, double *val, int *nnz, int *singularOut);
    void GetIdp(int32_t *out);

    LevelView View0() const { return L[0].view(); }
    size_t FieldSizeU() const { return (size_t)(Nx + 1) * Ny * Nz; }
    size_t FieldSizeV() const { return (size_t)Nx * (Ny + 1) * Nz; }
    size_t FieldSizeW() const { return dim == 3 ? (size_t)Nx * Ny * (Nz + 1) : 0; }
    size_t Cells() const { return (size_t)Nx * Ny * Nz; }

  private:
    friend struct Batch;
    void BuildHierarchy();
    void RefillHierarchy();
    void BuildPairData();
    void EnsureIdp();
    void AllocVectors();
    double ReadSlot(int s);
    void ReadSlots(int s, int count);
    // Solve A x = b (b in this->b, grid layout); the solution ends in *xOut (xa or xb). Fills out->iters/rel_res.
    // guess: the initial iterate (grid layout, zero off the unknowns; may be xb), else zero. refNorm > 0: stop at
    // ||r|| < tol max(||b||, refNorm), and when ||b|| <= tol refNorm already the answer is the guess (or zero)
    // (SolveEigenPressure, PressureSettings.h:411-427).
    int Solve(double tol, double **xOut, nb_result *out, const double *guess = nullptr, double refNorm = 0.0);
    int SolveMixed(double tol, double **xOut, nb_result *out, const double *guess, double refNorm);
    // The relative tolerance asked of each FP32 inner solve for a solve to `tol`: opt.inner_tol, or sqrt(tol) (at
    // least 1e-6) when tol is below opt.inner_tol^2, so that two refinement passes reach it (measured on the 2D
    // 128^2 box to 1e-10: 2 passes and 13 iterations instead of 3 and 17, 1.09 instead of 1.40 ms).
    // Solves since the last layout change that dropped the captured graphs. The graphs (use_graphs) are captured
    // from a layout's second solve on: a first solve on a new shape launches plainly, since capturing and
    // instantiating them costs more than they save once (measured: a 4-slot server whose requests all change shape
    // served 393 solves/s without them, 225 with them).
    int solvesOnShape = 0;
    int GraphMode() const { return solvesOnShape > 0 ? opt.use_graphs : 0; }
    double InnerTol(double tol) const
    {
        return tol >= opt.inner_tol * opt.inner_tol ? opt.inner_tol : std::max(1e-6, std::sqrt(tol));
    }
    // The squared residual, in the inner solve's scaling (rr0 = the pass's starting residual there, sfac the FP64 ->
    // inner factor), at which a pass's CG loop stops: the pass's relative reduction. A pass whose reduction already
    // reaches the outer tolerance (the last one) stops between a tenth and a half of it instead: no further than a
    // tenth (a warm start's last pass starts far below the first pass's residual), and not above a half, so that the
    // solution's distance from the exact one does not hang on where the last CG step lands just under the tolerance.
    static double InnerTarget(double rr0, double innerTol, double tol, double bn2, double sfac)
    {
        const double t = rr0 * innerTol * innerTol, q = tol * sfac, goal = q * q * bn2;
        if (t > goal) return t;
        return std::min(std::max(t, 0.01 * goal), 0.25 * goal);
    }
    void BuildSolveGraph();
    int SolveFP64(double tol, double **xOut, nb_result *out, const double *guess, double refNorm);
    // the initial residual of the guess, and the tolerance the refNorm floor turns `tol` into; false: nothing to do
    bool StartFrom(const double *guess, double refNorm, double tol, double bn2, double *tolEff);
    template <typename T> void VCycle(int l, T *r, T *e);
    // red-black sweeps before / after the coarse correction on level l (stretched levels take stretched_sweeps)
    int PreSweeps(int l) const { return std::max(1, L[l].stretched ? opt.stretched_sweeps : opt.pre_sweeps); }
    int PostSweeps(int l) const { return std::max(1, L[l].stretched ? opt.stretched_sweeps : opt.post_sweeps); }
    // the FP32 cell-pair kernels serve this level (its du is built)
    bool PairLevel(int l) const { return opt.pair_kernels && L[l].du.p != nullptr; }
    // the FP32 vectors of this level are colour-split and its V-cycle runs the split kernels
    bool Split(int l) const { return L[l].sRS != 0; }
    // FP32 elements of a level-0 vector (the split layout pads its rows)
    size_t VecLen0() const { return L[0].VecLen(); }
    void VCyclePairs(int l, float *r, float *e);
    void VCycleSplit(int l, float *r, float *e);
    void UploadTables();
    void AssignSplit();
    void BuildTailLists();
    // copyRR: end with the copy of r.r to the host (not inside the device-side loop)
    template <typename T> void IterBody(T *x, T *r, T *z, T *p0, T *p1, T *q, bool exact, bool copyRR = true);
    template <typename T> void BuildLoop(IterGraph *G, T *x, T *r, T *z, T *p0, T *p1, T *q, bool exact);
    template <typename T>
    int RunPCG(T *x, T *r, T *z, T *p0, T *p1, T *q, double rrStart, double rrTarget, int maxIt, bool exact,
               double *rrEnd);
};

// nb_noalloc.cu: the IDP numbering of device-resident cell types with scratch in a fixed per-device array (no
// allocation); at most kNoAllocMaxLines interior lines. idp and *n are device memory; asynchronous on st.
constexpr int kNoAllocMaxLines = 1 << 18;
void NumberUnknownsNoAlloc(int device, int dim, int Nx, int Ny, int Nz, const uint8_t *types, int32_t *idp,
                           int32_t *n, cudaStream_t st);

// FLIP's re-labelling from particles (nb_relabel.cu): the labels FLIP{2,3}D::UpdateFluidCells leaves, on `st`, no
// allocation. skipped (device, may be null) gets the number of particles outside the labels.
size_t RelabelScratchBytes(int dim, int Nx, int Ny, int Nz);
void UpdateFluidCellsDevice(int dim, int Nx, int Ny, int Nz, double ox, double oy, double oz, double dh,
                            const double *px, const double *py, const double *pz, long long count, long long stride,
                            uint8_t *cellTypes, void *scratch, size_t scratchBytes, unsigned long long *skipped,
                            cudaStream_t st);

// Boundary-condition replay (nb_bc.cu): the reference's lists as leveled device write programs.
struct BcReplay;
// Checks the lists on the host (every index inside its field); throws InputError on a bad list.
// The x groups of a stretched level's coarsening from its n interior x widths: left to right, two cells form one
// coarse cell when together they are at most 1.5 coarse y/z cells wide (twice yzMin), else a cell stays whole.
// count gets each group's cell count (1 or 2).
void PlanXGroups(const double *w, int n, double yzMin, std::vector<int> &count);
// Those groups as the transfer maps of LevelView::xp (nf + 2 entries, the rings included) and xr (Nc entries), with
// the coarse cell widths (Nc entries, each ring as wide as its neighbour); false (nothing written) when the groups
// are the regular pairing of every axis.
bool XMaps(const double *w, int nf, double yzMin, int &Nc, std::vector<double> &size, std::vector<int> &xp,
           std::vector<int> &xr);

void CheckBcLists(const nb_bc_lists &lists);
// The level of each operation of the two replays, in list order (solid faces of u, v, w, prescribed entries, copies;
// ring entries), on the host.
void PlanBcLevels(const nb_bc_lists &lists, std::vector<int> &velocity, std::vector<int> &pressure);
// The checked, levelled lists on the current device.
BcReplay *CreateBcReplay(int device, const nb_bc_lists &lists);
void DestroyBcReplay(BcReplay *b);
int BcLevels(const BcReplay &b, int pressure);
int BcDevice(const BcReplay &b);
void EnforceVelocityDevice(BcReplay &b, double *u, double *v, double *w, const double *prescValues, cudaStream_t st);
void EnforcePressureDevice(BcReplay &b, double *p, const double *ringValues, cudaStream_t st);

} // namespace nb
