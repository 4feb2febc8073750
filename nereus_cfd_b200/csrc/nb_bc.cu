// Boundary-condition replay on the device: MAC::EnforceVelocityBC and MAC::EnforcePressureBC (src/MAC.cpp:811-865)
// from the lists MAC::BuildBoundaryLists makes on the host (src/MAC.cpp:613-1090), so that a stepping loop can keep
// u, v, w and p on the device between its sub-steps. The fields come out bit for bit as the reference's serial
// replay leaves them.
//
// The reference replays, in order: zeros on solidFaceList[c]; the boundary velocity function's values on
// prescribedList (when the scene has one); copies f[dst] = f[src] on copyList (a corner copies from an edge that
// copied from a face, so the order matters); ApplyOutflowFlux; and, for p, ringList (zero, prescribed value or copy).
// Here the writes of one call form a program of (field, dst, source) operations, grouped once, at creation, into
// levels: an operation goes one level after the last earlier write of its destination, after every earlier read of
// its destination, and after the last earlier write of its source. Operations of one level touch distinct
// destinations and read nothing another operation of the level writes, so each level is one race-free scatter launch
// and the levels in turn give exactly the sequential result. Leaving out the prescribed writes (no velocity
// function) keeps that true: a removed write only ever added ordering.
//
// ApplyOutflowFlux sums sign * f * area over the inlet and the outflow faces in list order; one block forms the
// products in parallel, one thread adds them in the reference's order (so the correction rounds as the reference's
// does), and the block applies it. The prescribed values (the tinyexpr boundary functions) are evaluated by the
// caller on the host, as the reference does, and passed per call as a device array in list order.
#include "nb_solver.h"

#include <cstdint>
#include <memory>
#include <unordered_map>
#include <vector>

namespace nb
{

namespace
{

constexpr int kBcThreads = 256;
constexpr int kFluxThreads = 512;

struct BcOp
{
    int32_t comp; // field: 0 u, 1 v, 2 w (velocity); 0 p (pressure)
    int32_t dst;
    int32_t src;  // >= 0: copy f[src]
    int32_t val;  // src < 0, val >= 0: values[val]; both < 0: zero
};

__global__ void __launch_bounds__(kBcThreads)
    k_bc_level(const BcOp *__restrict__ ops, int n, double *f0, double *f1, double *f2,
               const double *__restrict__ values, int nullValuesZero)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
    {
        const BcOp o = ops[q];
        double *f = o.comp == 0 ? f0 : (o.comp == 1 ? f1 : f2);
        if (o.src >= 0)
            f[o.dst] = f[o.src];
        else if (o.val >= 0)
        {
            if (values) f[o.dst] = values[o.val];
            else if (nullValuesZero) f[o.dst] = 0.0;
        }
        else
            f[o.dst] = 0.0;
    }
}

struct FluxFaces
{
    const int32_t *comp, *index, *outer; // inlet faces first (outer unused), then the outflow faces
    const double *area, *sign;
    int nin, nout;
    double aOut;                         // sum of the outflow areas, in list order (host)
};

__global__ void __launch_bounds__(kFluxThreads) k_bc_outflow(FluxFaces ff, double *f0, double *f1, double *f2,
                                                             double *prod)
{
    __shared__ double delta;
    const int n = ff.nin + ff.nout;
    for (int q = threadIdx.x; q < n; q += blockDim.x)
    {
        const double *f = ff.comp[q] == 0 ? f0 : (ff.comp[q] == 1 ? f1 : f2);
        prod[q] = ff.sign[q] * f[ff.index[q]] * ff.area[q];
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double qIn = 0.0, qOut = 0.0;
        for (int q = 0; q < ff.nin; q++) qIn -= prod[q];
        for (int q = ff.nin; q < n; q++) qOut += prod[q];
        delta = (qIn - qOut) / ff.aOut;
    }
    __syncthreads();
    for (int q = ff.nin + threadIdx.x; q < n; q += blockDim.x)
    {
        double *f = ff.comp[q] == 0 ? f0 : (ff.comp[q] == 1 ? f1 : f2);
        const double v = f[ff.index[q]] + ff.sign[q] * delta;
        f[ff.index[q]] = v;
        f[ff.outer[q]] = v;
    }
}

// Levels of a sequential write program (see the top of this file); returns the operations sorted by level (stable),
// the start of each level and each operation's level in program order.
void LevelProgram(const std::vector<BcOp> &seq, std::vector<BcOp> &sorted, std::vector<int> &start,
                  std::vector<int> &level)
{
    std::unordered_map<long long, int> lastWrite, lastRead;
    lastWrite.reserve(seq.size() * 2);
    lastRead.reserve(seq.size());
    level.assign(seq.size(), 0);
    int nlev = 0;
    auto key = [](int c, int i) { return ((long long)c << 32) | (unsigned)i; };
    for (size_t q = 0; q < seq.size(); q++)
    {
        const BcOp &o = seq[q];
        int l = 0;
        auto after = [&](const std::unordered_map<long long, int> &m, long long k) {
            auto it = m.find(k);
            if (it != m.end() && it->second + 1 > l) l = it->second + 1;
        };
        const long long kd = key(o.comp, o.dst);
        after(lastWrite, kd);
        after(lastRead, kd);
        if (o.src >= 0)
        {
            const long long ks = key(o.comp, o.src);
            after(lastWrite, ks);
            auto it = lastRead.find(ks);
            if (it == lastRead.end() || it->second < l) lastRead[ks] = l;
        }
        lastWrite[kd] = l;
        level[q] = l;
        if (l + 1 > nlev) nlev = l + 1;
    }
    start.assign(nlev + 1, 0);
    for (size_t q = 0; q < seq.size(); q++) start[level[q] + 1]++;
    for (int l = 0; l < nlev; l++) start[l + 1] += start[l];
    std::vector<int> fill(start.begin(), start.end() - 1);
    sorted.resize(seq.size());
    for (size_t q = 0; q < seq.size(); q++) sorted[fill[level[q]]++] = seq[q];
}

} // namespace

struct BcReplay
{
    int device = 0;
    int dim = 3;
    int npresc = 0, nring = 0;
    DevArray<BcOp> vel, pres;
    std::vector<int> velStart, presStart;
    DevArray<int32_t> fluxI;  // comp | index | outer, each nin + nout
    DevArray<double> fluxD;   // area | sign | products
    FluxFaces ff{};
};

struct BcHost
{
    int dim = 3, npresc = 0, nring = 0, nin = 0, nout = 0;
    std::vector<BcOp> vel, pres;
    std::vector<int> velStart, presStart;
    std::vector<int> velLevel, presLevel; // each operation's level, in list order
    std::vector<int32_t> fluxI;
    std::vector<double> fluxD;
    double aOut = 0.0;
};

namespace
{
void CheckIndex(long long i, long long size, const char *what)
{
    if (i < 0 || i >= size) throw InputError(std::string(what) + " index outside its field");
}
} // namespace

static BcHost BuildBcHost(const nb_bc_lists &L)
{
    if (L.dim != 2 && L.dim != 3) throw InputError("dim must be 2 or 3");
    const long long nz = L.dim == 3 ? L.Nz : 1;
    if (L.Nx < 1 || L.Ny < 1 || nz < 1) throw InputError("bad sizes");
    const long long Nx = L.Nx, Ny = L.Ny;
    const long long sizes[3] = {(Nx + 1) * Ny * nz, Nx * (Ny + 1) * nz, L.dim == 3 ? Nx * Ny * (nz + 1) : 0};
    const long long pSize = Nx * Ny * nz;
    for (long long s : sizes)
        if (s >= (1ll << 31)) throw InputError("fields of at most 2^31 - 1 entries");
    auto counts_ok = [](int n, const void *p) { return n == 0 || (n > 0 && p); };
    for (int c = 0; c < 3; c++)
        if (!counts_ok(L.nsolid[c], L.solid[c])) throw InputError("solid face list");
    if (!counts_ok(L.npresc, L.presc_comp) || !counts_ok(L.npresc, L.presc_index)) throw InputError("prescribed list");
    if (!counts_ok(L.ncopy, L.copy_comp) || !counts_ok(L.ncopy, L.copy_dst) || !counts_ok(L.ncopy, L.copy_src))
        throw InputError("copy list");
    if (!counts_ok(L.nring, L.ring_dst) || !counts_ok(L.nring, L.ring_kind) || !counts_ok(L.nring, L.ring_src))
        throw InputError("ring list");
    if (!counts_ok(L.ninlet, L.inlet_comp) || !counts_ok(L.ninlet, L.inlet_index) ||
        !counts_ok(L.ninlet, L.inlet_area) || !counts_ok(L.ninlet, L.inlet_sign))
        throw InputError("inlet faces");
    if (!counts_ok(L.noutflow, L.outflow_comp) || !counts_ok(L.noutflow, L.outflow_index) ||
        !counts_ok(L.noutflow, L.outflow_outer) || !counts_ok(L.noutflow, L.outflow_area) ||
        !counts_ok(L.noutflow, L.outflow_sign))
        throw InputError("outflow faces");
    const int ncomp = L.dim == 3 ? 3 : 2;
    auto comp_ok = [&](int c) {
        if (c < 0 || c >= ncomp) throw InputError("velocity component out of range");
        return c;
    };

    std::vector<BcOp> seq;
    seq.reserve((size_t)L.nsolid[0] + L.nsolid[1] + L.nsolid[2] + L.npresc + L.ncopy);
    for (int c = 0; c < 3; c++)
        for (int q = 0; q < L.nsolid[c]; q++)
        {
            comp_ok(c);
            CheckIndex(L.solid[c][q], sizes[c], "solid face");
            seq.push_back({c, L.solid[c][q], -1, -1});
        }
    for (int q = 0; q < L.npresc; q++)
    {
        const int c = comp_ok(L.presc_comp[q]);
        CheckIndex(L.presc_index[q], sizes[c], "prescribed");
        seq.push_back({c, L.presc_index[q], -1, q});
    }
    for (int q = 0; q < L.ncopy; q++)
    {
        const int c = comp_ok(L.copy_comp[q]);
        CheckIndex(L.copy_dst[q], sizes[c], "copy destination");
        CheckIndex(L.copy_src[q], sizes[c], "copy source");
        seq.push_back({c, L.copy_dst[q], L.copy_src[q], -1});
    }
    std::vector<BcOp> pseq;
    pseq.reserve(L.nring);
    for (int q = 0; q < L.nring; q++)
    {
        CheckIndex(L.ring_dst[q], pSize, "ring destination");
        const int kind = L.ring_kind[q];
        if (kind < 0 || kind > 2) throw InputError("ring kind must be 0, 1 or 2");
        if (kind == 2) CheckIndex(L.ring_src[q], pSize, "ring source");
        pseq.push_back({0, L.ring_dst[q], kind == 2 ? L.ring_src[q] : -1, kind == 1 ? q : -1});
    }
    const int nin = L.ninlet, nout = L.noutflow;
    std::vector<int32_t> fi(3 * (size_t)(nin + nout), 0);
    std::vector<double> fd(3 * (size_t)(nin + nout), 0.0);
    double aOut = 0.0;
    for (int q = 0; q < nin + nout; q++)
    {
        const bool out = q >= nin;
        const int r = out ? q - nin : q;
        const int c = comp_ok(out ? L.outflow_comp[r] : L.inlet_comp[r]);
        const int idx = out ? L.outflow_index[r] : L.inlet_index[r];
        CheckIndex(idx, sizes[c], "flux face");
        fi[q] = c;
        fi[(nin + nout) + q] = idx;
        if (out)
        {
            CheckIndex(L.outflow_outer[r], sizes[c], "flux face outer");
            fi[2 * (nin + nout) + q] = L.outflow_outer[r];
            aOut += L.outflow_area[r];
        }
        fd[q] = out ? L.outflow_area[r] : L.inlet_area[r];
        fd[(nin + nout) + q] = out ? L.outflow_sign[r] : L.inlet_sign[r];
    }

    BcHost h;
    h.dim = L.dim;
    h.npresc = L.npresc;
    h.nring = L.nring;
    LevelProgram(seq, h.vel, h.velStart, h.velLevel);
    LevelProgram(pseq, h.pres, h.presStart, h.presLevel);
    h.fluxI.swap(fi);
    h.fluxD.swap(fd);
    h.nin = nin;
    h.nout = nout;
    h.aOut = aOut;
    return h;
}

static BcReplay *CreateBcReplay(int device, const BcHost &h)
{
    std::unique_ptr<BcReplay> b(new BcReplay);
    b->device = device;
    b->dim = h.dim;
    b->npresc = h.npresc;
    b->nring = h.nring;
    b->velStart = h.velStart;
    b->presStart = h.presStart;
    if (!h.vel.empty()) b->vel.upload(h.vel.data(), h.vel.size(), 0);
    if (!h.pres.empty()) b->pres.upload(h.pres.data(), h.pres.size(), 0);
    const int n = h.nin + h.nout;
    if (n > 0)
    {
        b->fluxI.upload(h.fluxI.data(), h.fluxI.size(), 0);
        b->fluxD.upload(h.fluxD.data(), h.fluxD.size(), 0);
    }
    NB_CK(cudaStreamSynchronize(0));
    b->ff.comp = b->fluxI.p;
    b->ff.index = b->fluxI.p ? b->fluxI.p + n : nullptr;
    b->ff.outer = b->fluxI.p ? b->fluxI.p + 2 * n : nullptr;
    b->ff.area = b->fluxD.p;
    b->ff.sign = b->fluxD.p ? b->fluxD.p + n : nullptr;
    b->ff.nin = h.nin;
    b->ff.nout = h.nout;
    b->ff.aOut = h.aOut;
    return b.release();
}

void CheckBcLists(const nb_bc_lists &lists) { (void)BuildBcHost(lists); }

void PlanBcLevels(const nb_bc_lists &lists, std::vector<int> &velocity, std::vector<int> &pressure)
{
    BcHost h = BuildBcHost(lists);
    velocity.swap(h.velLevel);
    pressure.swap(h.presLevel);
}

BcReplay *CreateBcReplay(int device, const nb_bc_lists &lists) { return CreateBcReplay(device, BuildBcHost(lists)); }

void DestroyBcReplay(BcReplay *b) { delete b; }

int BcLevels(const BcReplay &b, int pressure) { return (int)(pressure ? b.presStart : b.velStart).size() - 1; }

int BcDevice(const BcReplay &b) { return b.device; }

namespace
{
void RunLevels(const DevArray<BcOp> &ops, const std::vector<int> &start, double *f0, double *f1, double *f2,
               const double *values, int nullValuesZero, cudaStream_t st)
{
    for (size_t l = 0; l + 1 < start.size(); l++)
    {
        const int n = start[l + 1] - start[l];
        if (n <= 0) continue;
        int blocks = (n + kBcThreads - 1) / kBcThreads;
        if (blocks > 148 * 8) blocks = 148 * 8;
        NB_COUNT_LAUNCH();
        k_bc_level<<<blocks, kBcThreads, 0, st>>>(ops.p + start[l], n, f0, f1, f2, values, nullValuesZero);
    }
}
} // namespace

void EnforceVelocityDevice(BcReplay &b, double *u, double *v, double *w, const double *prescValues, cudaStream_t st)
{
    if (!u || !v || (b.dim == 3 && !w)) throw InputError("null velocity field");
    RunLevels(b.vel, b.velStart, u, v, w, prescValues, 0, st);
    if (b.ff.nout > 0 && b.ff.aOut > 0.0)
    {
        NB_COUNT_LAUNCH();
        k_bc_outflow<<<1, kFluxThreads, 0, st>>>(b.ff, u, v, w, b.fluxD.p + 2 * (b.ff.nin + b.ff.nout));
    }
    NB_CK(cudaGetLastError());
}

void EnforcePressureDevice(BcReplay &b, double *p, const double *ringValues, cudaStream_t st)
{
    if (!p) throw InputError("null pressure field");
    RunLevels(b.pres, b.presStart, p, p, p, ringValues, 1, st);
    NB_CK(cudaGetLastError());
}

} // namespace nb
