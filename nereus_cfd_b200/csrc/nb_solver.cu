// Host orchestration of the B200 pressure projection (see nb_solver.h).
//
// The pressure step follows PressureSolver3D::SolveScheme + ProjectPressure (src/Methods/PPESolver/
// PressureSolver3D.cpp:279-328, 417-438): ring, right-hand side, compatibility, solve, level, scatter, ring,
// projection. The solve replaces Eigen's diagonal-preconditioned CG (PressureSettings.h:386-481) by a matrix-free
// multigrid-preconditioned CG, in FP64 or as FP32 MG-PCG inside FP64 iterative refinement.
#include "nb_solver.h"

#include <algorithm>
#include <type_traits>

namespace nb
{

// ---------------------------------------------------------------------------------------------------------------
// levels
// ---------------------------------------------------------------------------------------------------------------
LevelView LevelData::view() const
{
    LevelView v{};
    v.dim = dim;
    v.Nx = Nx;
    v.Ny = Ny;
    v.Nz = Nz;
    v.cells = cells;
    if (dim == 3)
    {
        v.sI = (long long)Nx * Nz;
        v.sJ = Nz;
        v.nLines = (Ny - 2) * (Nx - 2);
        v.lineLen = Nz - 2;
        v.lineDiv = Nx - 2;
    }
    else
    {
        v.sI = Nx;
        v.sJ = 1;
        v.nLines = Ny - 2;
        v.lineLen = Nx - 2;
        v.lineDiv = 1;
    }
    if (v.nLines < 0 || v.lineLen <= 0) v.nLines = 0;
    if (v.lineDiv <= 0) v.lineDiv = 1;
    v.fastLen = std::max(0, dim == 3 ? Nz - 2 : Nx - 2);
    v.midLen = std::max(0, dim == 3 ? Nx - 2 : Ny - 2);
    v.slowLen = dim == 3 ? std::max(0, Ny - 2) : 1;
    {
        // reduction launches march far enough along the slow axis to be about two waves of 8 blocks per SM (their
        // partial sums stay few); the other stencil launches take one step per block
        const long long perPlane = (long long)((v.fastLen + kTileF - 1) / kTileF) * ((v.midLen + kTileM - 1) / kTileM);
        const long long target = 148 * 16;
        long long chunk = perPlane > 0 ? (v.slowLen * perPlane + target - 1) / target : 1;
        v.slowChunk = (int)std::max(1LL, std::min<long long>(chunk, std::max(1, v.slowLen)));
    }
    v.code = code.p;
    v.types = types.p;
    v.sRS = sRS;
    v.sPS = sPS;
    v.sHalf = sHalf;
    v.act = sRS && actTiles ? act.p : nullptr;
    v.actTiles = sRS ? actTiles : 0;
    v.stretched = stretched ? 1 : 0;
    v.gamma = gamma;
    v.xp = dxp;
    v.xr = dxr;
    for (int a = 0; a < 3; a++)
    {
        v.w[a] = dw[a];
        v.g[a] = dg[a];
        v.w32[a] = dw32[a];
        v.ig32[a] = dig32[a];
    }
    return v;
}

template <> float *LevelData::r<float>() { return r32.p; }
template <> double *LevelData::r<double>() { return r64.p; }
template <> float *LevelData::e<float>() { return e32.p; }
template <> double *LevelData::e<double>() { return e64.p; }
template <> float *LevelData::res<float>() { return res32.p; }
template <> double *LevelData::res<double>() { return res64.p; }

// Every level's spacing tables (Width and FaceGap in FP64, Width and 1/FaceGap in FP32, per axis) packed into one
// pinned staging buffer and sent in one copy into one device array; the level views point into it. A layout
// change thus costs one transfer instead of twelve per level. The staging buffer is rewritten only by the next
// layout, which starts with the stream idle.
void Context::UploadTables()
{
    auto pad = [](size_t b) { return (b + 15) & ~size_t(15); };
    size_t bytes = 0;
    for (const LevelData &Lv : L)
    {
        for (int a = 0; a < 3; a++)
            bytes += 2 * pad(Lv.w[a].size() * 8) + 2 * pad(Lv.g[a].size() * 8);
        bytes += pad(Lv.xp.size() * 4) + pad(Lv.xr.size() * 4);
    }
    if (bytes > tablesHostCap)
    {
        if (tablesHost) NB_CK(cudaFreeHost(tablesHost));
        tablesHost = nullptr;
        tablesHostCap = 0;
        NB_CK(cudaMallocHost((void **)&tablesHost, bytes));
        tablesHostCap = bytes;
    }
    tables.alloc(bytes);
    size_t off = 0;
    auto put = [&](const void *src, size_t n) {
        if (n) std::memcpy(tablesHost + off, src, n);
        const size_t at = off;
        off += pad(n);
        return at;
    };
    struct Off
    {
        size_t w, g, w32, ig32;
    };
    std::vector<Off> offs(L.size() * 3);
    for (size_t l = 0; l < L.size(); l++)
        for (int a = 0; a < 3; a++)
        {
            const LevelData &Lv = L[l];
            Off &o = offs[l * 3 + a];
            o.w = put(Lv.w[a].data(), Lv.w[a].size() * 8);
            o.g = put(Lv.g[a].data(), Lv.g[a].size() * 8);
            float *w32 = (float *)(tablesHost + off);
            for (size_t q = 0; q < Lv.w[a].size(); q++) w32[q] = (float)Lv.w[a][q];
            o.w32 = off;
            off += pad(Lv.w[a].size() * 4);
            float *ig32 = (float *)(tablesHost + off);
            for (size_t q = 0; q < Lv.g[a].size(); q++) ig32[q] = (float)(1.0 / Lv.g[a][q]);
            o.ig32 = off;
            off += pad(Lv.g[a].size() * 4);
        }
    std::vector<size_t> xOff(2 * L.size());
    for (size_t l = 0; l < L.size(); l++)
    {
        xOff[2 * l] = put(L[l].xp.data(), L[l].xp.size() * 4);
        xOff[2 * l + 1] = put(L[l].xr.data(), L[l].xr.size() * 4);
    }
    NB_CK(cudaMemcpyAsync(tables.p, tablesHost, off, cudaMemcpyHostToDevice, st));
    for (size_t l = 0; l < L.size(); l++)
        for (int a = 0; a < 3; a++)
        {
            const Off &o = offs[l * 3 + a];
            L[l].dw[a] = (const double *)(tables.p + o.w);
            L[l].dg[a] = (const double *)(tables.p + o.g);
            L[l].dw32[a] = (const float *)(tables.p + o.w32);
            L[l].dig32[a] = (const float *)(tables.p + o.ig32);
        }
    for (size_t l = 0; l < L.size(); l++)
    {
        L[l].dxp = L[l].xp.empty() ? nullptr : (const int *)(tables.p + xOff[2 * l]);
        L[l].dxr = L[l].xr.empty() ? nullptr : (const int *)(tables.p + xOff[2 * l + 1]);
    }
}

// Coarse padded tables of one axis: interior widths summed in pairs, the ring mirroring its neighbour
// (MAC::AddRing), padded and gapped like MAC::PadTable / MAC::GapTable.
static void CoarseAxis(const std::vector<double> &wFine, int Nf, int Nc, std::vector<double> &wOut,
                       std::vector<double> &gOut)
{
    // wFine is padded: Width(n) = wFine[n + 1], n = -1..Nf
    const int nf = Nf - 2, m = Nc - 2;
    std::vector<double> size(Nc);
    for (int I = 1; I <= m; I++)
    {
        const int a = 2 * I - 1, b = 2 * I;
        size[I] = wFine[a + 1] + (b <= nf ? wFine[b + 1] : 0.0);
    }
    size[0] = size[1];
    size[Nc - 1] = size[m];
    wOut.resize(Nc + 2);
    for (int q = -1; q <= Nc; q++) wOut[q + 1] = size[q < 0 ? 0 : (q >= Nc ? Nc - 1 : q)];
    gOut.resize(Nc + 1);
    for (int q = -1; q <= Nc - 1; q++)
    {
        const double a = size[q < 0 ? 0 : (q >= Nc ? Nc - 1 : q)];
        const double b = size[q + 1 >= Nc ? Nc - 1 : q + 1];
        gOut[q + 1] = 0.5 * (a + b);
    }
}

// x groups of stretched coarsening (declared with their rule in nb_solver.h)
void PlanXGroups(const double *w, int n, double yzMin, std::vector<int> &count)
{
    const double target = 1.5 * 2.0 * yzMin;
    count.clear();
    for (int j = 0; j < n;)
    {
        const bool two = j + 1 < n && w[j] + w[j + 1] <= target;
        count.push_back(two ? 2 : 1);
        j += two ? 2 : 1;
    }
}

bool XMaps(const double *w, int nf, double yzMin, int &Nc, std::vector<double> &size, std::vector<int> &xp,
           std::vector<int> &xr)
{
    std::vector<int> first, count; // interior groups: first fine cell (grid index), children
    PlanXGroups(w, nf, yzMin, count);
    for (size_t g = 0, j = 1; g < count.size(); j += count[g], g++) first.push_back((int)j);
    const int m = (int)first.size();
    bool regular = true;
    for (int g = 0; g < m; g++)
        if (count[g] != 2 && !(g == m - 1 && first[g] == nf)) regular = false;
    if (regular) return false;
    if (nf + 2 > 0x7FFF) return false; // the maps pack indices in 15 bits
    Nc = m + 2;
    size.assign(Nc, 0.0);
    for (int g = 0; g < m; g++) size[g + 1] = w[first[g] - 1] + (count[g] == 2 ? w[first[g]] : 0.0);
    size[0] = size[1];
    size[Nc - 1] = size[m];
    // fine j -> parent, other contributor, single; the rings map onto the rings
    xp.assign(nf + 2, 0);
    xp[0] = 0 | (0 << 15) | (1 << 30);
    xp[nf + 1] = (Nc - 1) | ((Nc - 1) << 15) | (1 << 30);
    xr.assign(Nc, 0);
    xr[0] = 0;
    xr[Nc - 1] = nf + 1;
    for (int g = 0; g < m; g++)
    {
        const int J = g + 1;
        if (count[g] == 1) xp[first[g]] = J | (J << 15) | (1 << 30);
        else
        {
            xp[first[g]] = J | ((J - 1) << 15);
            xp[first[g] + 1] = J | ((J + 1) << 15);
        }
        const bool before = g > 0 && count[g - 1] == 2, after = g + 1 < m && count[g + 1] == 2;
        xr[J] = first[g] | ((count[g] == 2) << 15) | (before << 16) | (after << 17);
    }
    return true;
}

// The x groups of a stretched 3D level's next coarsening (XMaps with the level's thinnest interior y or z width),
// with the coarse level's padded x tables (as CoarseAxis makes them) and its extent; false: the regular pairing.
static bool XGroups(const LevelData &F, int &Nc, std::vector<double> &wOut, std::vector<double> &gOut,
                    std::vector<int> &xp, std::vector<int> &xr)
{
    double yz = 1e300;
    for (int a = 1; a <= 2; a++)
    {
        const int n = (a == 1 ? F.Ny : F.Nz) - 2;
        for (int q = 0; q < n; q++) yz = std::min(yz, F.w[a][q + 2]);
    }
    std::vector<double> size;
    if (!XMaps(F.w[0].data() + 2, F.Nx - 2, yz, Nc, size, xp, xr)) return false;
    wOut.resize(Nc + 2);
    for (int q = -1; q <= Nc; q++) wOut[q + 1] = size[q < 0 ? 0 : (q >= Nc ? Nc - 1 : q)];
    gOut.resize(Nc + 1);
    for (int q = -1; q <= Nc - 1; q++)
    {
        const double a = size[q < 0 ? 0 : (q >= Nc ? Nc - 1 : q)];
        const double b = size[q + 1 >= Nc ? Nc - 1 : q + 1];
        gOut[q + 1] = 0.5 * (a + b);
    }
    return true;
}

void Context::BuildHierarchy()
{
    // the previous levels lend their device arrays to the new ones of the same index (a DevArray keeps its
    // allocation when the new size fits), so a new shape allocates only where it outgrows the old
    std::vector<LevelData> old = std::move(L);
    L.clear();
    L.reserve(32);
    auto take = [&](size_t l) {
        LevelData X = l < old.size() ? std::move(old[l]) : LevelData();
        for (int a = 0; a < 3; a++) { X.w[a].clear(); X.g[a].clear(); }
        X.xp.clear();
        X.xr.clear();
        X.dxp = X.dxr = nullptr;
        return X;
    };
    {
        LevelData L0 = take(0);
        L0.dim = dim;
        L0.Nx = Nx;
        L0.Ny = Ny;
        L0.Nz = Nz;
        L0.cells = (long long)Nx * Ny * Nz;
        L0.stretched = nonuniform;
        L0.gamma = 1.0;
        for (int a = 0; a < 3; a++) { L0.w[a] = wt[a]; L0.g[a] = gt[a]; }
        L0.types.upload(layout.data(), layout.size(), st);
        L0.code.alloc(layout.size());
        L.push_back(std::move(L0));
    }
    const int maxLevels = std::max(1, opt.max_levels);
    while ((int)L.size() < maxLevels)
    {
        LevelData &F = L.back();
        const int nx = F.Nx - 2, ny = F.Ny - 2, nz = dim == 3 ? F.Nz - 2 : 1;
        const int mn = dim == 3 ? std::min(nx, std::min(ny, nz)) : std::min(nx, ny);
        const long long interior = (long long)nx * ny * nz;
        // down to 4 .. 7 cells a side (at most a few hundred unknowns), solved by sweeps in the shared-memory tail:
        // one level more, of a handful of unknowns, made no difference to the iteration counts measured and only
        // lengthened the tail's serial phases
        if (mn < 8 || interior <= 64) break;
        LevelData C = take(L.size());
        C.dim = dim;
        // x kept whole where a pair would be much wider than the coarse y/z cells (not on the coarse end's levels,
        // whose transfers pair every axis)
        const bool grouped = dim == 3 && F.stretched && opt.x_groups && F.cells > (long long)opt.tail_cells &&
                             XGroups(F, C.Nx, C.w[0], C.g[0], F.xp, F.xr);
        if (!grouped) C.Nx = (nx + 1) / 2 + 2;
        C.Ny = (ny + 1) / 2 + 2;
        C.Nz = dim == 3 ? (nz + 1) / 2 + 2 : 1;
        C.cells = (long long)C.Nx * C.Ny * C.Nz;
        C.stretched = F.stretched;
        C.gamma = F.gamma * (dim == 3 ? 2.0 : 1.0);
        if (!grouped) CoarseAxis(F.w[0], F.Nx, C.Nx, C.w[0], C.g[0]);
        CoarseAxis(F.w[1], F.Ny, C.Ny, C.w[1], C.g[1]);
        if (dim == 3) CoarseAxis(F.w[2], F.Nz, C.Nz, C.w[2], C.g[2]);
        else { C.w[2] = F.w[2]; C.g[2] = F.g[2]; }
        C.types.alloc((size_t)C.cells);
        C.code.alloc((size_t)C.cells);
        L.push_back(std::move(C));
    }
    // the levels' tables, then their cell types and codes, level by level
    UploadTables();
    LaunchBuildCodes(L[0].view(), L[0].code.p, st);
    for (size_t l = 1; l < L.size(); l++)
    {
        LaunchCoarsenTypes(L[l - 1].view(), L[l].view(), L[l].types.p, st);
        LaunchBuildCodes(L[l].view(), L[l].code.p, st);
    }
    NB_CK(cudaGetLastError());
    // The tail: the first level from which every coarser level has at most opt.tail_cells cells and all of them fit
    // in one block's shared memory in the solver's precision.
    const bool mixed = opt.precision == NB_PRECISION_MIXED;
    tailStart = (int)L.size();
    std::vector<LevelView> views;
    for (auto &Lv : L) views.push_back(Lv.view());
    for (int l = (int)L.size() - 1; l >= 0; l--)
    {
        const int nl = (int)L.size() - l;
        if (nl > kMaxTailLevels || L[l].cells > (long long)opt.tail_cells) break;
        if (std::max(L[l].Nx, std::max(L[l].Ny, L[l].Nz)) > 1023) break; // the tail packs i, j, k in 10 bits each
        const size_t bytes = mixed ? TailSmemBytes<float>(&views[l], nl) : TailSmemBytes<double>(&views[l], nl);
        if (bytes > kTailMaxSmem) break;
        tailStart = l;
    }
    if (tailStart < (int)L.size())
    {
        const bool ok = mixed ? PrepareTail<float>(kTailMaxSmem) : PrepareTail<double>(kTailMaxSmem);
        if (!ok) tailStart = (int)L.size();
    }
    AssignSplit();
    BuildPairData();
    BuildTailLists();
    NB_CK(cudaGetLastError());
}

// The colour-split levels (pair_kernels = 2, mixed precision): the uniform 3D levels with Nz even above the coarse
// end, as long as every finer level is one too (a level's transfers read and write the next coarser level in either
// layout, the grid-layout kernels only the grid layout). A stretched grid keeps the cell-pair kernels: its
// per-cell coefficients make the split kernels compute-bound (measured slower on the stretched cylinder).
void Context::AssignSplit()
{
    const bool on = opt.precision == NB_PRECISION_MIXED && opt.pair_kernels == 2 && !nonuniform;
    bool finer = true;
    for (size_t l = 0; l < L.size(); l++)
    {
        LevelData &Lv = L[l];
        Lv.sRS = Lv.sPS = 0;
        Lv.sHalf = 0;
        const bool s = on && finer && (int)l < tailStart && l + 1 < L.size() && PairLevelShape(Lv.view());
        if (s)
        {
            Lv.sRS = ((Lv.Nz / 2) + 3) & ~3;
            Lv.sPS = Lv.Nx * Lv.sRS;
            Lv.sHalf = ((long long)Lv.Ny * Lv.sPS + 63) & ~63LL; // each colour starts 256-byte aligned
        }
        finer = s;
    }
}

// The per-level bytes of the cell-pair and colour-split kernels: diagonal units (codes on a stretched split level)
// and the prolongation's moved weights.
void Context::BuildPairData()
{
    // the FP32 kernels' diagonal units (mixed precision: the inner solve runs in FP32)
    for (auto &Lv : L)
    {
        const LevelView v = Lv.view();
        if (opt.precision == NB_PRECISION_MIXED && opt.pair_kernels && PairLevelShape(v))
        {
            if (Lv.sRS)
            {
                PrepareSplitKernels();
                Lv.du.alloc((size_t)(2 * Lv.sHalf));
                Lv.du.zero(st); // the padding
                LaunchBuildDu(v, Lv.du.p, st);
                if (opt.skip_idle_tiles)
                {
                    Lv.actTiles = SplitActivityTiles(v);
                    Lv.act.alloc((size_t)Lv.Ny * Lv.actTiles);
                    LaunchSplitActivity(v, Lv.du.p, Lv.act.p, Lv.actTiles, st);
                }
                else
                {
                    Lv.actTiles = 0;
                    Lv.act.release();
                }
            }
            else
            {
                Lv.du.alloc((size_t)Lv.cells);
                LaunchBuildDu(v, Lv.du.p, st);
            }
        }
        else Lv.du.release();
    }
    for (size_t l = 0; l < L.size(); l++)
    {
        if (L[l].du.p && l + 1 < L.size())
        {
            if (L[l].sRS)
            {
                L[l].pext.alloc((size_t)L[l].sHalf);
                L[l].pext.zero(st);
            }
            else L[l].pext.alloc((size_t)L[l].cells);
            LaunchBuildPext(L[l].view(), L[l + 1].view(), L[l].pext.p, st);
        }
        else L[l].pext.release();
    }
}

// A new layout with the hierarchy's shape (sizes and spacing tables) unchanged: the cell types, codes and pair bytes of
// every level are rebuilt in the arrays they have; pointers, tail and captured iterations stay as they are.
void Context::RefillHierarchy()
{
    L[0].types.upload(layout.data(), layout.size(), st);
    LaunchBuildCodes(L[0].view(), L[0].code.p, st);
    for (size_t l = 1; l < L.size(); l++)
    {
        LaunchCoarsenTypes(L[l - 1].view(), L[l].view(), L[l].types.p, st);
        LaunchBuildCodes(L[l].view(), L[l].code.p, st);
    }
    BuildPairData();
    BuildTailLists();
    NB_CK(cudaGetLastError());
}

// The tail levels' lists of unknowns by colour (they follow the cell types).
void Context::BuildTailLists()
{
    if (tailStart >= (int)L.size())
    {
        tailLists.release();
        tailCounts.release();
        return;
    }
    std::vector<LevelView> views;
    for (size_t q = (size_t)tailStart; q < L.size(); q++) views.push_back(L[q].view());
    tailLists.alloc((size_t)TailListEntries(views.data(), (int)views.size()));
    tailCounts.alloc(2 * kMaxTailLevels);
    LaunchTailLists(views.data(), (int)views.size(), tailLists.p, tailCounts.p, st);
}

void Context::AllocVectors()
{
    const bool mixed = opt.precision == NB_PRECISION_MIXED;
    for (size_t l = 0; l < L.size(); l++)
    {
        LevelData &Lv = L[l];
        const size_t c = (size_t)Lv.cells;
        const bool last = l + 1 == L.size();
        if (mixed)
        {
            const size_t c32 = Lv.VecLen(); // zeroed whole: the split layout's padding stays zero
            Lv.r32.alloc(c32); Lv.r32.zero(st);
            Lv.e32.alloc(c32); Lv.e32.zero(st);
            if (!last) { Lv.res32.alloc(c32); Lv.res32.zero(st); }
            Lv.r64.release(); Lv.e64.release(); Lv.res64.release();
        }
        else
        {
            Lv.r64.alloc(c); Lv.r64.zero(st);
            Lv.e64.alloc(c); Lv.e64.zero(st);
            if (!last) { Lv.res64.alloc(c); Lv.res64.zero(st); }
            Lv.r32.release(); Lv.e32.release(); Lv.res32.release();
        }
    }
    const size_t c = Cells();
    b.alloc(c); b.zero(st);
    xa.alloc(c); xa.zero(st);
    xb.alloc(c); xb.zero(st);
    if (mixed)
    {
        const size_t c32 = VecLen0();
        for (auto &a : p32) { a.alloc(c32); a.zero(st); }
        q32.alloc(c32); q32.zero(st);
        x32.alloc(c32); x32.zero(st);
        for (auto &a : p64) a.release();
        q64.release();
    }
    else
    {
        for (auto &a : p64) { a.alloc(c); a.zero(st); }
        q64.alloc(c); q64.zero(st);
        for (auto &a : p32) a.release();
        q32.release();
        x32.release();
    }
}

// ---------------------------------------------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------------------------------------------
Context::Context(const nb_options &o) : opt(o)
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
    arrays.Init(device, st);
    red.maxBlocks = 1 << 16; // partial sums per reduction launch (the tile grids stay well below)
    partials.alloc((size_t)red.maxBlocks * 4);
    slots.alloc(S_COUNT);
    slots.zero(st);
    counter.alloc(1);
    counter.zero(st);
    iter.alloc(1);
    iter.zero(st);
    passes.alloc(1);
    passes.zero(st);
    red.partials = partials.p;
    red.out = slots.p;
    red.counter = counter.p;
    NB_CK(cudaMallocHost((void **)&hostSlots, sizeof(double) * S_COUNT));
    NB_CK(cudaEventCreate(&ev0));
    NB_CK(cudaEventCreate(&ev1));
}

Context::~Context()
{
    if (st) cudaStreamSynchronize(st);
    for (auto &g : graphs) g.Release();
    ReleaseSolveGraph();
    if (cst) cudaStreamSynchronize(cst);
    for (cudaEvent_t e : evPool) cudaEventDestroy(e);
    if (evP) cudaEventDestroy(evP);
    if (evPDone) cudaEventDestroy(evPDone);
    if (cst) cudaStreamDestroy(cst);
    if (hostSlots) cudaFreeHost(hostSlots);
    if (tablesHost) cudaFreeHost(tablesHost);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    L.clear();
    arrays.st = nullptr; // the arrays still to go are freed after the stream, on the legacy one (nothing runs now)
    if (ownStream && st) cudaStreamDestroy(st);
}

// ---- per-kernel timing: events from a pool, bracketing launches of the selected kernel ids ----
void Context::ProfBegin(int id, double bytes, int launches)
{
    if (profQuiet || !(profMask >> id & 1u)) return;
    cudaEvent_t a;
    if (capturing)
    {
        NB_CK(cudaEventCreate(&a));
        capturing->events.push_back(a);
    }
    else
    {
        if (evUsed + 2 > evPool.size())
            for (int q = 0; q < 256; q++)
            {
                cudaEvent_t e;
                NB_CK(cudaEventCreate(&e));
                evPool.push_back(e);
            }
        a = evPool[evUsed++];
    }
    profA = a;
    // inside a capture, an external record becomes an event-record node that every replay executes
    NB_CK(capturing ? cudaEventRecordWithFlags(profA, st, cudaEventRecordExternal) : cudaEventRecord(profA, st));
    profOpen = id;
    profBytes = bytes;
    profLaunches = launches;
}

void Context::ProfEnd(int launches)
{
    if (profQuiet || profOpen < 0) return;
    if (launches >= 0) profLaunches = launches;
    cudaEvent_t b;
    if (capturing)
    {
        NB_CK(cudaEventCreate(&b));
        capturing->events.push_back(b);
    }
    else
        b = evPool[evUsed++];
    NB_CK(capturing ? cudaEventRecordWithFlags(b, st, cudaEventRecordExternal) : cudaEventRecord(b, st));
    (capturing ? capturing->prof : prof).push_back({profOpen, profA, b, profBytes, profLaunches});
    profOpen = -1;
}

static void Accumulate(const std::vector<Context::ProfRecord> &recs, Context::ProfTotal *tot)
{
    for (const Context::ProfRecord &r : recs)
    {
        float m = 0.0f;
        NB_CK(cudaEventElapsedTime(&m, r.a, r.b));
        tot[r.id].launches += r.launches;
        tot[r.id].ms += m;
        tot[r.id].bytes += r.bytes;
    }
}

// Resolve the stream-launch records into the totals and recycle their events (the stream must be idle).
void Context::ProfFlush()
{
    if (prof.empty()) return;
    NB_CK(cudaStreamSynchronize(st));
    Accumulate(prof, profTot);
    prof.clear();
    evUsed = 0;
}

void Context::ProfClear()
{
    prof.clear();
    evUsed = 0;
    profOpen = -1;
    for (auto &t : profTot) t = ProfTotal();
}

void Context::ProfRead(int id, int *launches, double *ms, double *bytesPerLaunch)
{
    ProfFlush();
    const ProfTotal &t = profTot[id];
    *launches = (int)t.launches;
    *ms = t.ms;
    *bytesPerLaunch = t.launches ? t.bytes / (double)t.launches : 0.0;
}

void Context::IterGraph::Release()
{
    if (loopExec) cudaGraphExecDestroy(loopExec);
    if (loop) cudaGraphDestroy(loop);
    loopExec = nullptr;
    loop = nullptr;
    loopFailed = false;
    if (exec) cudaGraphExecDestroy(exec);
    if (g) cudaGraphDestroy(g);
    for (cudaEvent_t e : events) cudaEventDestroy(e);
    exec = nullptr;
    g = nullptr;
    events.clear();
    prof.clear();
    mask = 0;
}

double Context::ReadSlot(int s)
{
    NB_CK(cudaMemcpyAsync(hostSlots + s, slots.p + s, sizeof(double), cudaMemcpyDeviceToHost, st));
    NB_CK(cudaStreamSynchronize(st));
    return hostSlots[s];
}

void Context::ReadSlots(int s, int count)
{
    NB_CK(cudaMemcpyAsync(hostSlots + s, slots.p + s, sizeof(double) * count, cudaMemcpyDeviceToHost, st));
    NB_CK(cudaStreamSynchronize(st));
}

// Every byte <= 5 (the six cell types), eight at a time: a byte b >= 6 has bit 7 set in b + 0x7A or in b itself.
static bool TypesInRange(const uint8_t *t, size_t n)
{
    const uint64_t k7A = 0x7A7A7A7A7A7A7A7AULL, k80 = 0x8080808080808080ULL;
    size_t c = 0;
    uint64_t bad = 0;
    for (; c + 8 <= n; c += 8)
    {
        uint64_t x;
        std::memcpy(&x, t + c, 8);
        bad |= (x | ((x & 0x7F7F7F7F7F7F7F7FULL) + k7A)) & k80;
    }
    for (; c < n; c++) bad |= t[c] > 5 ? 1u : 0u;
    return bad == 0;
}

void Context::SetLayout(int dim_, int Nx_, int Ny_, int Nz_, const uint8_t *types, const double *const width[3],
                        const double *const gap[3], int nonUniform, double dh_)
{
    if (dim_ != 2 && dim_ != 3) throw InputError("dim must be 2 or 3");
    if (dim_ == 2) Nz_ = 1;
    if (Nx_ < 2 || Ny_ < 2 || Nz_ < 1 || (dim_ == 3 && Nz_ < 2)) throw InputError("grid too small");
    if (!types || !width || !gap) throw InputError("null layout pointer");
    for (int a = 0; a < (dim_ == 3 ? 3 : 2); a++)
        if (!width[a] || !gap[a]) throw InputError("null spacing table");
    if (!nonUniform && !(dh_ > 0.0)) throw InputError("uniform grid needs dh > 0");
    const size_t cells = (size_t)Nx_ * Ny_ * Nz_;
    if (!TypesInRange(types, cells)) throw InputError("cell type out of range");
    const int N[3] = {Nx_, Ny_, Nz_};
    bool same = built && dim_ == dim && Nx_ == Nx && Ny_ == Ny && Nz_ == Nz && (nonUniform != 0) == nonuniform &&
                dh_ == dh && layout.size() == cells && std::memcmp(layout.data(), types, cells) == 0;
    for (int a = 0; a < 3 && same; a++)
    {
        const size_t nw = (size_t)N[a] + 2, ng = (size_t)N[a] + 1;
        if (a == 2 && dim_ == 2) continue;
        same = wt[a].size() == nw && gt[a].size() == ng && std::memcmp(wt[a].data(), width[a], nw * 8) == 0 &&
               std::memcmp(gt[a].data(), gap[a], ng * 8) == 0;
    }
    if (same) return; // PressureLayoutChanged: nothing moved
    ArrayPoolScope pooled(&arrays);
    // the same shape (sizes, spacing tables, dh): only the cell types moved, the hierarchy is refilled in place
    bool shapeSame = built && dim_ == dim && Nx_ == Nx && Ny_ == Ny && Nz_ == Nz &&
                     (nonUniform != 0) == nonuniform && dh_ == dh && layout.size() == cells;
    for (int a = 0; a < 3 && shapeSame; a++)
    {
        const size_t nw = (size_t)N[a] + 2, ng = (size_t)N[a] + 1;
        if (a == 2 && dim_ == 2) continue;
        shapeSame = wt[a].size() == nw && gt[a].size() == ng && std::memcmp(wt[a].data(), width[a], nw * 8) == 0 &&
                    std::memcmp(gt[a].data(), gap[a], ng * 8) == 0;
    }
    // a uniform grid of the same sizes at another dh: the hierarchy keeps its shape (the FP32 levels see gamma, not
    // dh); the spacing tables and the scale are replaced in the arrays they have, so the captured iterations stay
    const bool rescale = !shapeSame && built && !nonUniform && !nonuniform && dim_ == dim && Nx_ == Nx &&
                         Ny_ == Ny && Nz_ == Nz && layout.size() == cells;
    NB_CK(cudaStreamSynchronize(st));
    const bool wasSingular = singular;
    built = false;
    idpValid = false;
    layout.assign(types, types + cells);
    if (rescale)
    {
        dh = dh_;
        scale = 1.0 / (dh * dh); // MatrixScale3D (PressureSolver3D.cpp:34-37)
        for (int a = 0; a < (dim == 3 ? 3 : 2); a++)
        {
            std::vector<double> w(width[a], width[a] + N[a] + 2), g(gap[a], gap[a] + N[a] + 1);
            for (double x : w)
                if (!(x > 0.0) || !std::isfinite(x)) throw InputError("width table entries must be positive");
            for (double x : g)
                if (!(x > 0.0) || !std::isfinite(x)) throw InputError("gap table entries must be positive");
            wt[a] = w;
            gt[a] = g;
        }
        if (dim == 2)
        {
            wt[2].assign(3, wt[0][1]);
            gt[2].assign(2, wt[0][1]);
        }
        for (int a = 0; a < 3; a++) { L[0].w[a] = wt[a]; L[0].g[a] = gt[a]; }
        for (size_t l = 1; l < L.size(); l++)
        {
            LevelData &F = L[l - 1], &C = L[l];
            CoarseAxis(F.w[0], F.Nx, C.Nx, C.w[0], C.g[0]);
            CoarseAxis(F.w[1], F.Ny, C.Ny, C.w[1], C.g[1]);
            if (dim == 3) CoarseAxis(F.w[2], F.Nz, C.Nz, C.w[2], C.g[2]);
            else { C.w[2] = F.w[2]; C.g[2] = F.g[2]; }
        }
        UploadTables(); // same sizes: the same device array
        ReleaseSolveGraph();                     // its refinement step holds the old scale
        solvesOnShape = 0;
        RefillHierarchy();
    }
    else if (shapeSame)
        RefillHierarchy();
    else
    {
        for (auto &g : graphs) g.Release(); // they hold the old hierarchy's pointers
        ReleaseSolveGraph();
        solvesOnShape = 0;
        dim = dim_;
        Nx = Nx_;
        Ny = Ny_;
        Nz = Nz_;
        nonuniform = nonUniform != 0;
        dh = dh_;
        scale = nonuniform ? 1.0 : 1.0 / (dh * dh); // MatrixScale3D (PressureSolver3D.cpp:34-37)
        for (int a = 0; a < 3; a++)
        {
            if (a == 2 && dim == 2)
            {
                const double w0 = width[2] ? width[2][1] : (width[0] ? width[0][1] : 1.0);
                wt[2].assign(3, w0);
                gt[2].assign(2, w0);
                continue;
            }
            wt[a].assign(width[a], width[a] + N[a] + 2);
            gt[a].assign(gap[a], gap[a] + N[a] + 1);
            for (double x : wt[a])
                if (!(x > 0.0) || !std::isfinite(x)) throw InputError("width table entries must be positive");
            for (double x : gt[a])
                if (!(x > 0.0) || !std::isfinite(x)) throw InputError("gap table entries must be positive");
        }
        BuildHierarchy();
    }
    // the system size and the singular flag, counted on the device (the IDP numbering waits until it is asked for)
    LaunchCountUnknowns(L[0].view(), red, S_RES, st);
    ReadSlots(S_RES, 2);
    n = (int)hostSlots[S_RES];
    singular = hostSlots[S_RES + 1] == 0.0;
    if ((shapeSame || rescale) && singular != wasSingular)
    {
        for (auto &g : graphs) g.Release(); // the iteration's kernels depend on the flag
        ReleaseSolveGraph();
        solvesOnShape = 0;
    }
    hostSlots[S_NUNK] = (double)n;
    NB_CK(cudaMemcpyAsync(slots.p + S_NUNK, hostSlots + S_NUNK, sizeof(double), cudaMemcpyHostToDevice, st));
    AllocVectors();
    NB_CK(cudaStreamSynchronize(st));
    built = true;
}

// ---------------------------------------------------------------------------------------------------------------
// multigrid V-cycle and PCG
// ---------------------------------------------------------------------------------------------------------------
// The levels below level 0 of one V-cycle under one bracket of the per-kernel timing (NB_K_COARSE): their dozens
// of short kernels then overlap their dependent launches as in an unprofiled solve, where a bracket of events around
// each (a few us apiece) would both inflate and serialise them.
template <typename T> void Context::CoarseBracket(int l, T *r, T *e)
{
    const long long n0 = g_launches.load();
    ProfBegin(NB_K_COARSE, 0.0);
    const bool quiet = profQuiet;
    profQuiet = true;
    VCycle<T>(l, r, e);
    profQuiet = quiet;
    ProfEnd((int)(g_launches.load() - n0));
}

template <typename T> void Context::VCycle(int l, T *r, T *e)
{
    LevelData &Lv = L[l];
    const LevelView v = Lv.view();
    const double s = sizeof(T), cells = (double)Lv.cells;
    // kernel id and algorithmic bytes per launch (each array touched once) for the finest level's kernels
    auto prof = [&](int id, double bytesPerCell) {
        ProfBegin(l == 0 ? id : NB_K_COARSE, l == 0 ? bytesPerCell * cells : 0.0);
    };
    if (l == tailStart)
    {
        std::vector<LevelView> views;
        for (size_t q = (size_t)l; q < L.size(); q++) views.push_back(L[q].view());
        prof(NB_K_COARSE, 0.0);
        LaunchTail<T>(views.data(), (int)views.size(), r, e, PreSweeps(l), PostSweeps(l), opt.coarse_sweeps,
                      tailLists.p, tailCounts.p, st);
        ProfEnd();
        return;
    }
    if (l + 1 == (int)L.size())
    {
        prof(NB_K_COARSE, 0.0);
        LaunchCoarseSolve<T>(v, r, e, opt.coarse_sweeps, st);
        ProfEnd();
        return;
    }
    if constexpr (std::is_same<T, float>::value)
    {
        if (Split(l))
        {
            VCycleSplit(l, r, e);
            return;
        }
        if (PairLevel(l))
        {
            VCyclePairs(l, r, e);
            return;
        }
    }
    const int pre = PreSweeps(l), post = PostSweeps(l);
    const double half = (3.0 * s + 1.0) / 2.0; // one red-black sweep reads e, r, types and writes e: 3s + 1
    prof(NB_K_SMOOTH0, 2.0 * s + 1.0);
    LaunchSmoothFirst<T>(v, r, e, st);
    ProfEnd();
    prof(NB_K_SMOOTH0, half);
    LaunchSmooth<T>(v, r, e, 1, st);
    ProfEnd();
    for (int q = 1; q < pre; q++)
    {
        prof(NB_K_SMOOTH0, half);
        LaunchSmooth<T>(v, r, e, 0, st);
        ProfEnd();
        prof(NB_K_SMOOTH0, half);
        LaunchSmooth<T>(v, r, e, 1, st);
        ProfEnd();
    }
    T *res = Lv.res<T>();
    prof(NB_K_RESIDUAL0, 3.0 * s + 1.0);
    LaunchLevelResidual<T>(v, r, e, res, st);
    ProfEnd();
    LevelData &Lc = L[l + 1];
    const LevelView vc = Lc.view();
    prof(NB_K_RESTRICT0, s + s / 8.0);
    LaunchRestrict<T>(v, vc, res, Lc.r<T>(), st);
    ProfEnd();
    if (l == 0) CoarseBracket<T>(l + 1, Lc.r<T>(), Lc.e<T>());
    else VCycle<T>(l + 1, Lc.r<T>(), Lc.e<T>());
    prof(NB_K_PROLONG0, 2.0 * s + s / 8.0 + 1.0);
    LaunchProlong<T>(v, vc, Lc.e<T>(), e, st);
    ProfEnd();
    for (int q = 0; q < post; q++)
    {
        prof(NB_K_SMOOTH0, half);
        LaunchSmooth<T>(v, r, e, 1, st);
        ProfEnd();
        prof(NB_K_SMOOTH0, half);
        LaunchSmooth<T>(v, r, e, 0, st);
        ProfEnd();
    }
}

// The V-cycle on a 3D FP32 level with the cell-pair kernels (nb_pairs.cu): the first red-black sweep from zero (one
// launch on a uniform level, a red and a black one on a stretched level), further sweeps one colour per launch, the
// residual, and the pair transfers.
void Context::VCyclePairs(int l, float *r, float *e)
{
    LevelData &Lv = L[l];
    const LevelView v = Lv.view();
    const bool stretched = v.stretched != 0;
    const double s = sizeof(float), cells = (double)Lv.cells;
    auto prof = [&](int id, double bytesPerCell) {
        ProfBegin(l == 0 ? id : NB_K_COARSE, l == 0 ? bytesPerCell * cells : 0.0);
    };
    const int pre = PreSweeps(l), post = PostSweeps(l);
    const double half = (3.0 * s + 1.0) / 2.0;
    if (stretched)
    {
        prof(NB_K_SMOOTH0, s + 1.0 + s / 2.0); // red from zero: reads r and codes, writes e
        LaunchPairHalfSt(v, r, e, 0, true, st);
        ProfEnd();
        prof(NB_K_SMOOTH0, half);
        LaunchPairHalfSt(v, r, e, 1, false, st);
        ProfEnd();
    }
    else
    {
        prof(NB_K_SMOOTH0, s + 1.0 + s); // reads r and du, writes e
        LaunchPairFirst(v, Lv.du.p, r, e, st);
        ProfEnd();
    }
    for (int q = 1; q < pre; q++)
        for (int c = 0; c < 2; c++)
        {
            prof(NB_K_SMOOTH0, half);
            if (stretched) LaunchPairHalfSt(v, r, e, c, false, st);
            else LaunchPairHalf(v, Lv.du.p, r, e, c, st);
            ProfEnd();
        }
    float *res = Lv.res<float>();
    prof(NB_K_RESIDUAL0, 3.0 * s + 1.0);
    if (stretched) LaunchPairResidualSt(v, r, e, res, st);
    else LaunchPairResidual(v, Lv.du.p, r, e, res, st);
    ProfEnd();
    LevelData &Lc = L[l + 1];
    const LevelView vc = Lc.view();
    prof(NB_K_RESTRICT0, s + s / 8.0);
    LaunchPairRestrict(v, vc, Lv.pext.p, res, Lc.r<float>(), st);
    ProfEnd();
    if (l == 0) CoarseBracket<float>(l + 1, Lc.r<float>(), Lc.e<float>());
    else VCycle<float>(l + 1, Lc.r<float>(), Lc.e<float>());
    prof(NB_K_PROLONG0, 2.0 * s + s / 8.0 + 1.0);
    LaunchPairProlong(v, vc, Lv.pext.p, Lc.e<float>(), e, st);
    ProfEnd();
    for (int q = 0; q < post; q++)
        for (int c = 1; c >= 0; c--)
        {
            prof(NB_K_SMOOTH0, half);
            const bool dot = l == 0 && q + 1 == post && c == 0; // z is final: r.z for CG here (IterBody skips its own)
            if (stretched)
            {
                if (dot) LaunchPairHalfStDot(v, r, e, c, red, iter.p, S_RZ0, S_RZ1, st);
                else LaunchPairHalfSt(v, r, e, c, false, st);
            }
            else
            {
                if (dot) LaunchPairHalfDot(v, Lv.du.p, r, e, c, red, iter.p, S_RZ0, S_RZ1, st);
                else LaunchPairHalf(v, Lv.du.p, r, e, c, st);
            }
            ProfEnd();
        }
}

// The V-cycle on a colour-split level (nb_split.cu): the first sweep from zero in one launch, further sweeps one
// colour per launch, the residual and the transfers on the
// red cells (the black residual after a black half-sweep is zero; the post-smoothing's black half replaces the black
// values without reading them), and on level 0 the (r.z, z, r) sums of the last sweep, black then red.
void Context::VCycleSplit(int l, float *r, float *e)
{
    LevelData &Lv = L[l];
    const LevelView v = Lv.view();
    const double s = sizeof(float), cells = (double)Lv.cells;
    auto prof = [&](int id, double bytesPerCell) {
        ProfBegin(l == 0 ? id : NB_K_COARSE, l == 0 ? bytesPerCell * cells : 0.0);
    };
    const int pre = PreSweeps(l), post = PostSweeps(l);
    // one colour: reads the other colour, and r and the bytes of its own; writes its own
    const double half = (3.0 * s + 1.0) / 2.0;
    const uint8_t *du = Lv.du.p;
    prof(NB_K_SMOOTH0, 2.0 * s + 1.0); // reads r and the bytes, writes e
    LaunchSplitFirst(v, du, r, e, st);
    ProfEnd();
    for (int q = 1; q < pre; q++)
        for (int c = 0; c < 2; c++)
        {
            prof(NB_K_SMOOTH0, half);
            LaunchSplitHalf(v, du, r, e, c, st);
            ProfEnd();
        }
    float *res = Lv.res<float>();
    prof(NB_K_RESIDUAL0, (4.0 * s + 1.0) / 2.0); // reads e, and r and the bytes of red; writes red
    LaunchSplitResidual(v, du, r, e, res, st);
    ProfEnd();
    LevelData &Lc = L[l + 1];
    const LevelView vc = Lc.view();
    prof(NB_K_RESTRICT0, (s + 1.0) / 2.0 + s / 8.0);
    LaunchSplitRestrict(v, vc, Lv.pext.p, res, Lc.r<float>(), opt.transfer_kernels, st);
    ProfEnd();
    if (l == 0) CoarseBracket<float>(l + 1, Lc.r<float>(), Lc.e<float>());
    else VCycle<float>(l + 1, Lc.r<float>(), Lc.e<float>());
    prof(NB_K_PROLONG0, s + 0.5 + s / 8.0); // reads and writes red e, reads the red bytes and the coarse e
    LaunchSplitProlong(v, vc, Lv.pext.p, Lc.e<float>(), e, st);
    ProfEnd();
    for (int q = 0; q < post; q++)
    {
        // the black and the red half back to back: one pair of events around both (half the events' own cost)
        ProfBegin(l == 0 ? NB_K_SMOOTH0 : NB_K_COARSE, l == 0 ? 2.0 * half * cells : 0.0, 2);
        for (int c = 1; c >= 0; c--)
        {
            if (l == 0 && q + 1 == post) // z is final: r.z for CG here (IterBody skips its own)
                LaunchSplitHalfDot(v, du, r, e, c, c == 0, red, iter.p, S_RZ0, S_RZ1, S_RZB, st);
            else
                LaunchSplitHalf(v, du, r, e, c, st);
        }
        ProfEnd();
    }
}

// One CG iteration on level 0: z = V-cycle(r), r.z, p = z + beta p (and q = M p, p.q), x += alpha p, r -= alpha q,
// r.r copied to the host. The iteration number and the parity of the p buffers live on the device.
template <typename T> void Context::IterBody(T *x, T *r, T *z, T *p0, T *p1, T *q, bool exact, bool copyRR)
{
    const LevelView v0 = L[0].view();
    const double s = sizeof(T), cells = (double)Cells();
    const int sing = singular ? 1 : 0;
    VCycle<T>(0, r, z);
    if constexpr (std::is_same<T, float>::value)
    {
        if (Split(0)) // r.z came with the V-cycle's last sweep
        {
            ProfBegin(NB_K_PAPPLY, (4.0 * s + 1.0) * cells);
            LaunchSplitPApply(v0, L[0].du.p, z, p0, p1, q, red, slots.p, iter.p, S_RZ0, S_RZ1, S_NUNK, sing, S_PQ, st);
            ProfEnd();
            ProfBegin(NB_K_XR, 6.0 * s * cells);
            LaunchSplitLinXR(v0, (long long)VecLen0(), x, r, p0, p1, q, red, slots.p, iter.p, S_RZ0, S_RZ1, S_NUNK,
                             sing, S_PQ, S_RR, st);
            ProfEnd();
            if (copyRR)
                NB_CK(cudaMemcpyAsync(hostSlots + S_RR, slots.p + S_RR, sizeof(double), cudaMemcpyDeviceToHost, st));
            return;
        }
        if (PairLevel(0))
        {
            // r.z came with the V-cycle's last sweep unless level 0 is itself the coarse end (tail or single level)
            if (!(tailStart > 0 && L.size() > 1))
            {
                ProfBegin(NB_K_DOT, 2.0 * s * cells);
                LaunchLinDot(L[0].cells, r, z, red, iter.p, S_RZ0, S_RZ1, st);
                ProfEnd();
            }
            ProfBegin(NB_K_PAPPLY, (4.0 * s + 1.0) * cells);
            LaunchPairPApply(v0, L[0].du.p, z, p0, p1, q, red, slots.p, iter.p, S_RZ0, S_RZ1, S_NUNK, sing, S_PQ, st);
            ProfEnd();
            ProfBegin(NB_K_XR, 6.0 * s * cells);
            LaunchLinXR(L[0].cells, x, r, p0, p1, q, red, slots.p, iter.p, S_RZ0, S_RZ1, S_NUNK, sing, S_PQ, S_RR, st);
            ProfEnd();
            if (copyRR)
                NB_CK(cudaMemcpyAsync(hostSlots + S_RR, slots.p + S_RR, sizeof(double), cudaMemcpyDeviceToHost, st));
            return;
        }
    }
    ProfBegin(NB_K_DOT, 2.0 * s * cells);
    LaunchDot<T>(v0, r, z, red, iter.p, S_RZ0, S_RZ1, st);
    ProfEnd();
    ProfBegin(NB_K_PAPPLY, (4.0 * s + 1.0) * cells);
    LaunchUpdatePApply<T>(v0, z, p0, p1, q, red, slots.p, iter.p, S_RZ0, S_RZ1, S_NUNK, sing, S_PQ, exact ? 1 : 0, st);
    ProfEnd();
    ProfBegin(NB_K_XR, 6.0 * s * cells);
    LaunchUpdateXR<T>(v0, x, r, p0, p1, q, red, slots.p, iter.p, S_RZ0, S_RZ1, S_NUNK, sing, S_PQ, S_RR, st);
    ProfEnd();
    if (copyRR) NB_CK(cudaMemcpyAsync(hostSlots + S_RR, slots.p + S_RR, sizeof(double), cudaMemcpyDeviceToHost, st));
}

// The loop condition of the device-side CG loop, after an iteration's x/r update: go on while the iterations done are
// below the cap, r.r is above its target and finite (the host loop's test).
__global__ void k_loop_cond(cudaGraphConditionalHandle h, double *S, const int *it, int slotRR, int slotTgt,
                            int slotMax, int slotIts)
{
    const double rr = S[slotRR];
    const int n = *it;
    S[slotIts] = (double)n;
    const bool go = n < (int)S[slotMax] && rr > S[slotTgt] && isfinite(rr);
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

template <typename T> void Context::BuildLoop(IterGraph *G, T *x, T *r, T *z, T *p0, T *p1, T *q, bool exact)
{
    cudaGraph_t loop = nullptr;
    cudaGraphExec_t exec = nullptr;
    auto unavailable = [&]() {
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        if (loop) cudaGraphDestroy(loop);
        G->loopFailed = true;
    };
    cudaGraphConditionalHandle h = 0;
    if (cudaGraphCreate(&loop, 0) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&h, loop, 1, cudaGraphCondAssignDefault) != cudaSuccess)
        return unavailable();
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if (cudaGraphAddNode(&node, loop, nullptr, 0, &np) != cudaSuccess) return unavailable();
    cudaGraph_t body = np.conditional.phGraph_out[0];
    const long long before = g_launches.load();
    if (cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return unavailable();
    bool ok = true;
    try
    {
        IterBody<T>(x, r, z, p0, p1, q, exact, false);
        NB_COUNT_LAUNCH();
        k_loop_cond<<<1, 1, 0, st>>>(h, slots.p, iter.p, S_RR, S_TGT, S_MAXIT, S_ITS);
    }
    catch (...)
    {
        ok = false;
    }
    cudaGraph_t out = nullptr;
    if (cudaStreamEndCapture(st, &out) != cudaSuccess || !ok) return unavailable();
    if (cudaGraphInstantiate(&exec, loop, 0) != cudaSuccess) return unavailable();
    G->loop = loop;
    G->loopExec = exec;
    G->loopLaunches = g_launches.load() - before; // counted when run, not when recorded
    NB_COUNT_LAUNCHES(-G->loopLaunches);
}

template <typename T>
int Context::RunPCG(T *x, T *r, T *z, T *p0, T *p1, T *q, double rrStart, double rrTarget, int maxIt, bool exact,
                    double *rrEnd)
{
    NB_CK(cudaMemsetAsync(p0, 0, sizeof(T) * VecLen0(), st));
    NB_CK(cudaMemsetAsync(iter.p, 0, sizeof(int), st));
    if (GraphMode() >= 2 && profMask == 0)
    {
        // the whole loop on the device: one launch, one synchronisation
        IterGraph *L = &graphs[sizeof(T) == 8 ? 1 : 0];
        if (!L->loopExec && !L->loopFailed) BuildLoop<T>(L, x, r, z, p0, p1, q, exact);
        if (L->loopExec)
        {
            if (!(maxIt > 0 && rrStart > rrTarget))
            {
                *rrEnd = rrStart;
                return 0;
            }
            hostSlots[S_TGT] = rrTarget;
            hostSlots[S_MAXIT] = (double)maxIt;
            NB_CK(cudaMemcpyAsync(slots.p + S_TGT, hostSlots + S_TGT, 2 * sizeof(double), cudaMemcpyHostToDevice, st));
            NB_CK(cudaGraphLaunch(L->loopExec, st));
            NB_CK(cudaMemcpyAsync(hostSlots + S_RR, slots.p + S_RR, sizeof(double), cudaMemcpyDeviceToHost, st));
            NB_CK(cudaMemcpyAsync(hostSlots + S_ITS, slots.p + S_ITS, sizeof(double), cudaMemcpyDeviceToHost, st));
            NB_CK(cudaStreamSynchronize(st));
            NB_CK(cudaGetLastError());
            const int it = (int)hostSlots[S_ITS];
            NB_COUNT_LAUNCHES(it * L->loopLaunches);
            *rrEnd = hostSlots[S_RR];
            return it;
        }
    }
    IterGraph *G = nullptr;
    if (GraphMode())
    {
        G = &graphs[sizeof(T) == 8 ? 1 : 0];
        if (G->exec && G->mask != profMask) G->Release();
        if (!G->exec)
        {
            ProfFlush();
            const long long before = g_launches.load();
            NB_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            capturing = G;
            try
            {
                IterBody<T>(x, r, z, p0, p1, q, exact);
            }
            catch (...)
            {
                capturing = nullptr;
                cudaGraph_t dead = nullptr;
                cudaStreamEndCapture(st, &dead);
                if (dead) cudaGraphDestroy(dead);
                throw;
            }
            capturing = nullptr;
            NB_CK(cudaStreamEndCapture(st, &G->g));
            NB_CK(cudaGraphInstantiate(&G->exec, G->g, 0));
            G->mask = profMask;
            G->launches = g_launches.load() - before; // counted when replayed, not when recorded
            NB_COUNT_LAUNCHES(-G->launches);
        }
    }
    double rr = rrStart;
    int it = 0;
    while (it < maxIt && rr > rrTarget)
    {
        if (G)
        {
            NB_COUNT_LAUNCHES(G->launches);
            NB_CK(cudaGraphLaunch(G->exec, st));
            NB_CK(cudaStreamSynchronize(st));
            if (!G->prof.empty()) Accumulate(G->prof, profTot);
        }
        else
        {
            IterBody<T>(x, r, z, p0, p1, q, exact);
            NB_CK(cudaStreamSynchronize(st));
        }
        rr = hostSlots[S_RR];
        it++;
        if (!std::isfinite(rr)) break;
    }
    NB_CK(cudaGetLastError());
    *rrEnd = rr;
    return it;
}

bool Context::StartFrom(const double *guess, double refNorm, double tol, double bn2, double *tolEff)
{
    *tolEff = tol;
    bool go = true;
    if (refNorm > 0.0)
    {
        const double bn = std::sqrt(bn2);
        if (bn <= tol * refNorm) go = false; // nothing to solve: the answer is the guess (the increment is zero)
        else *tolEff = std::min(0.5, tol * refNorm / bn);
    }
    if (guess && guess != xa.p)
        NB_CK(cudaMemcpyAsync(xa.p, guess, sizeof(double) * Cells(), cudaMemcpyDeviceToDevice, st));
    return go;
}

// ---- the mixed solve as one graph (SolveMixed's loop on the device) ----
// Before the passes: ||b||^2 (the zero iterate's residual, in S_RES) is kept, no pass done yet, and the loop starts
// unless that residual already meets the tolerance (the host loop's test, sqrt(rr / bn2) <= tol, in the same order).
__global__ void k_mixed_init(cudaGraphConditionalHandle h, double *S, int *passes, int maxOuter)
{
    const double bn2 = S[S_RES];
    S[S_BN2] = bn2;
    S[S_INNER] = 0.0;
    *passes = 0;
    const bool go = bn2 > 0.0 && !(sqrt(bn2 / bn2) <= S[S_TOL]) && 0 < maxOuter && isfinite(bn2);
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

// A pass's CG targets: r.r down by inner_tol^2 from the unit-form residual of this pass, at most maxIt iterations;
// the CG loop's condition set to run (a handle's default value is applied when the whole graph is launched, not when
// an enclosing loop's body starts again).
__global__ void k_mixed_pass(cudaGraphConditionalHandle hInner, double *S, double sfac, int maxIt)
{
    // as Context::InnerTarget
    const double rr0 = S[S_RES] * sfac * sfac, innerTol = S[S_INTOL], q = S[S_TOL] * sfac;
    const double t = rr0 * innerTol * innerTol, goal = q * q * S[S_BN2];
    S[S_TGT] = t > goal ? t : fmin(fmax(t, 0.01 * goal), 0.25 * goal);
    S[S_MAXIT] = (double)maxIt;
    cudaGraphSetConditional(hInner, 1u);
}

// After a pass's refinement step: count it and its CG iterations; go on while the FP64 residual is above the
// tolerance, finite, and passes remain.
__global__ void k_mixed_cond(cudaGraphConditionalHandle h, double *S, int *passes, int maxOuter)
{
    const int n = *passes + 1;
    *passes = n;
    S[S_INNER] += S[S_ITS];
    const double rr = S[S_RES], bn2 = S[S_BN2];
    const bool go = !(sqrt(rr / bn2) <= S[S_TOL]) && n < maxOuter && isfinite(rr);
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

void Context::ReleaseSolveGraph()
{
    if (solveExec) cudaGraphExecDestroy(solveExec);
    if (solveGraph) cudaGraphDestroy(solveGraph);
    solveExec = nullptr;
    solveGraph = nullptr;
    solveFailed = false;
}

void Context::BuildSolveGraph()
{
    const LevelView v0 = L[0].view();
    const double sfac = -1.0 / scale;
    float *r32 = L[0].r32.p, *z32 = L[0].e32.p;
    const int maxOuter = std::max(1, opt.max_outer), maxIt = std::max(1, opt.max_iters);
    cudaGraph_t G = nullptr;
    auto unavailable = [&]() {
        cudaGetLastError();
        if (G) cudaGraphDestroy(G);
        solveGraph = nullptr;
        solveExec = nullptr;
        solveFailed = true;
    };
    // the sink nodes of the capture in progress on st
    auto sinks = [&](std::vector<cudaGraphNode_t> &out) {
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        if (cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &nd) != cudaSuccess) return false;
        out.assign(deps, deps + nd);
        return true;
    };
    auto endCapture = [&]() {
        cudaGraph_t g = nullptr;
        return cudaStreamEndCapture(st, &g) == cudaSuccess;
    };
    auto whileNode = [&](cudaGraph_t parent, const std::vector<cudaGraphNode_t> &deps, cudaGraphConditionalHandle h,
                         cudaGraph_t *body) {
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        if (cudaGraphAddNode(&node, parent, deps.empty() ? nullptr : deps.data(), deps.size(), &np) != cudaSuccess)
            return (cudaGraphNode_t) nullptr;
        *body = np.conditional.phGraph_out[0];
        return node;
    };
    cudaGraphConditionalHandle hOuter = 0, hInner = 0;
    if (cudaGraphCreate(&G, 0) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&hOuter, G, 0, cudaGraphCondAssignDefault) != cudaSuccess)
        return unavailable();
    const long long l0 = g_launches.load();
    std::vector<cudaGraphNode_t> deps;
    bool ok = true;
    // prologue: x = 0, the zero iterate's residual and ||b||^2, the loop's start
    if (cudaStreamBeginCaptureToGraph(st, G, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return unavailable();
    try
    {
        NB_CK(cudaMemsetAsync(xa.p, 0, xa.bytes(), st));
        if (Split(0)) LaunchSplitScaleSum(v0, b.p, r32, sfac, red, S_RES, st);
        else LaunchScaleSum<float>(L[0].cells, b.p, r32, sfac, red, S_RES, st);
        NB_COUNT_LAUNCH();
        k_mixed_init<<<1, 1, 0, st>>>(hOuter, slots.p, passes.p, maxOuter);
        ok = sinks(deps);
    }
    catch (...)
    {
        ok = false;
    }
    if (!endCapture() || !ok) return unavailable();
    const long long l1 = g_launches.load();
    cudaGraph_t outerBody = nullptr;
    cudaGraphNode_t outerNode = whileNode(G, deps, hOuter, &outerBody);
    if (!outerNode || cudaGraphConditionalHandleCreate(&hInner, outerBody, 1, cudaGraphCondAssignDefault) != cudaSuccess)
        return unavailable();
    // a pass: x32 = 0, p0 = 0, iteration 0, the targets
    if (cudaStreamBeginCaptureToGraph(st, outerBody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess)
        return unavailable();
    try
    {
        NB_CK(cudaMemsetAsync(x32.p, 0, x32.bytes(), st));
        NB_CK(cudaMemsetAsync(p32[0].p, 0, p32[0].bytes(), st));
        NB_CK(cudaMemsetAsync(iter.p, 0, sizeof(int), st));
        NB_COUNT_LAUNCH();
        k_mixed_pass<<<1, 1, 0, st>>>(hInner, slots.p, sfac, maxIt);
        ok = sinks(deps);
    }
    catch (...)
    {
        ok = false;
    }
    if (!endCapture() || !ok) return unavailable();
    const long long l2 = g_launches.load();
    cudaGraph_t innerBody = nullptr;
    cudaGraphNode_t innerNode = whileNode(outerBody, deps, hInner, &innerBody);
    if (!innerNode) return unavailable();
    // the CG iteration, its loop condition
    if (cudaStreamBeginCaptureToGraph(st, innerBody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess)
        return unavailable();
    try
    {
        IterBody<float>(x32.p, r32, z32, p32[0].p, p32[1].p, q32.p, false, false);
        NB_COUNT_LAUNCH();
        k_loop_cond<<<1, 1, 0, st>>>(hInner, slots.p, iter.p, S_RR, S_TGT, S_MAXIT, S_ITS);
    }
    catch (...)
    {
        ok = false;
    }
    if (!endCapture() || !ok) return unavailable();
    const long long l3 = g_launches.load();
    // the refinement step (iterates swapped by the pass count) and the outer condition
    std::vector<cudaGraphNode_t> afterInner(1, innerNode);
    if (cudaStreamBeginCaptureToGraph(st, outerBody, afterInner.data(), nullptr, 1,
                                      cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return unavailable();
    try
    {
        if (Split(0) && !nonuniform)
            LaunchSplitRefine64(v0, L[0].du.p, b.p, xa.p, x32.p, xb.p, r32, scale, sfac, red, S_RES, st, passes.p);
        else if (PairLevel(0) && !nonuniform && dim == 3)
            LaunchPairRefine64(v0, L[0].du.p, b.p, xa.p, x32.p, xb.p, r32, scale, sfac, red, S_RES, st, passes.p);
        else
            LaunchRefine64<float>(v0, b.p, xa.p, x32.p, xb.p, r32, scale, sfac, red, S_RES, st, passes.p);
        NB_COUNT_LAUNCH();
        k_mixed_cond<<<1, 1, 0, st>>>(hOuter, slots.p, passes.p, maxOuter);
    }
    catch (...)
    {
        ok = false;
    }
    if (!endCapture() || !ok) return unavailable();
    const long long l4 = g_launches.load();
    if (cudaGraphInstantiate(&solveExec, G, 0) != cudaSuccess) return unavailable();
    solveGraph = G;
    solvePrologLaunches = l1 - l0;
    solvePassLaunches = (l2 - l1) + (l4 - l3);
    solveIterLaunches = l3 - l2;
    NB_COUNT_LAUNCHES(-(l4 - l0)); // counted when run
}

int Context::SolveMixed(double tol, double **xOut, nb_result *out, const double *guess, double refNorm)
{
    if (GraphMode() >= 2 && profMask == 0 && !guess && !(refNorm > 0.0) && !solveFailed)
    {
        // the whole solve on the device: one launch, one synchronisation
        if (!solveExec) BuildSolveGraph();
        if (solveExec)
        {
            hostSlots[S_TOL] = tol;
            hostSlots[S_TOL + 1] = 0.0; // S_INNER, set on the device
            hostSlots[S_INTOL] = InnerTol(tol);
            static_assert(S_INTOL == S_TOL + 2, "the solve's host-set slots are contiguous");
            NB_CK(cudaMemcpyAsync(slots.p + S_TOL, hostSlots + S_TOL, 3 * sizeof(double), cudaMemcpyHostToDevice,
                                  st));
            NB_CK(cudaGraphLaunch(solveExec, st));
            int np = 0;
            NB_CK(cudaMemcpyAsync(hostSlots, slots.p, sizeof(double) * S_COUNT, cudaMemcpyDeviceToHost, st));
            NB_CK(cudaMemcpyAsync(&np, passes.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            NB_CK(cudaStreamSynchronize(st));
            NB_CK(cudaGetLastError());
            const double bn2 = hostSlots[S_BN2], rr64 = np > 0 ? hostSlots[S_RES] : bn2;
            const int inner = (int)hostSlots[S_INNER];
            NB_COUNT_LAUNCHES(solvePrologLaunches + np * solvePassLaunches + (long long)inner * solveIterLaunches);
            out->b_norm = std::sqrt(bn2);
            out->iters_outer = np;
            out->iters_inner = inner;
            out->rel_res = bn2 > 0.0 ? std::sqrt(rr64 / bn2) : 0.0;
            *xOut = (np & 1) ? xb.p : xa.p;
            return (bn2 > 0.0 && !(std::sqrt(rr64 / bn2) <= tol)) ? NB_NOT_CONVERGED : NB_OK;
        }
    }
    const LevelView v0 = L[0].view();
    const double sfac = -1.0 / scale;
    double *x = xa.p, *xo = xb.p;
    xa.zero(st);
    float *r32 = L[0].r32.p, *z32 = L[0].e32.p;
    ProfBegin(NB_K_REFINE, (8.0 + 4.0) * (double)Cells());
    if (Split(0)) LaunchSplitScaleSum(v0, b.p, r32, sfac, red, S_RES, st); // the residual of x = 0
    else LaunchScaleSum<float>(L[0].cells, b.p, r32, sfac, red, S_RES, st);
    ProfEnd();
    const double bn2 = ReadSlot(S_RES);
    out->b_norm = std::sqrt(bn2);
    int outer = 0, inner = 0, status = NB_OK;
    double rr64 = bn2, tolEff = tol;
    bool go = bn2 > 0.0;
    if (go)
    {
        go = StartFrom(guess, refNorm, tol, bn2, &tolEff);
        if (guess)
        {
            LaunchResidual64<float>(v0, b.p, x, r32, scale, sfac, red, S_RES, st);
            rr64 = ReadSlot(S_RES);
        }
    }
    if (go)
    {
        const int maxOuter = std::max(1, opt.max_outer);
        while (true)
        {
            if (std::sqrt(rr64 / bn2) <= tolEff) break;
            if (outer >= maxOuter || !std::isfinite(rr64)) { status = NB_NOT_CONVERGED; break; }
            x32.zero(st);
            double rrEnd = 0.0;
            const double rr0 = rr64 * sfac * sfac;
            const double tgt = InnerTarget(rr0, InnerTol(tolEff), tolEff, bn2, sfac);
            inner += RunPCG<float>(x32.p, r32, z32, p32[0].p, p32[1].p, q32.p, rr0, tgt,
                                   std::max(1, opt.max_iters), false, &rrEnd);
            ProfBegin(NB_K_REFINE, (8.0 + 4.0 + 8.0 + 1.0 + 8.0 + 4.0) * (double)Cells());
            if (Split(0) && !nonuniform)
                LaunchSplitRefine64(v0, L[0].du.p, b.p, x, x32.p, xo, r32, scale, sfac, red, S_RES, st);
            else if (PairLevel(0) && !nonuniform && dim == 3)
                LaunchPairRefine64(v0, L[0].du.p, b.p, x, x32.p, xo, r32, scale, sfac, red, S_RES, st);
            else
                LaunchRefine64<float>(v0, b.p, x, x32.p, xo, r32, scale, sfac, red, S_RES, st);
            ProfEnd();
            std::swap(x, xo);
            rr64 = ReadSlot(S_RES);
            outer++;
        }
    }
    out->iters_outer = outer;
    out->iters_inner = inner;
    out->rel_res = bn2 > 0.0 ? std::sqrt(rr64 / bn2) : 0.0;
    *xOut = x;
    return status;
}

int Context::SolveFP64(double tol, double **xOut, nb_result *out, const double *guess, double refNorm)
{
    const LevelView v0 = L[0].view();
    const double sfac = -1.0 / scale;
    double *x = xa.p;
    xa.zero(st);
    double *r = L[0].r64.p, *z = L[0].e64.p;
    ProfBegin(NB_K_REFINE, (8.0 + 8.0) * (double)Cells());
    LaunchScaleSum<double>(L[0].cells, b.p, r, sfac, red, S_RES, st); // the residual of x = 0
    ProfEnd();
    const double bn2 = ReadSlot(S_RES);
    out->b_norm = std::sqrt(bn2);
    int its = 0, status = NB_OK, restarts = 0;
    double rr = bn2, tolEff = tol;
    bool go = bn2 > 0.0;
    if (go)
    {
        go = StartFrom(guess, refNorm, tol, bn2, &tolEff);
        if (guess)
        {
            LaunchResidual64<double>(v0, b.p, x, r, scale, sfac, red, S_RES, st);
            rr = ReadSlot(S_RES);
        }
    }
    if (go)
    {
        const int maxIt = std::max(1, opt.max_iters) * std::max(1, opt.max_outer);
        while (true)
        {
            if (std::sqrt(rr / bn2) <= tolEff) break;
            if (its >= maxIt || restarts > 4 || !std::isfinite(rr)) { status = NB_NOT_CONVERGED; break; }
            double rrEnd = 0.0;
            // the recursive residual is driven a little below the target, then checked against the true one
            const double target = 0.25 * tolEff * tolEff * bn2 * sfac * sfac;
            its += RunPCG<double>(x, r, z, p64[0].p, p64[1].p, q64.p, rr * sfac * sfac, target, maxIt - its, true,
                                  &rrEnd);
            ProfBegin(NB_K_REFINE, (8.0 + 8.0 + 1.0 + 8.0) * (double)Cells());
            LaunchResidual64<double>(v0, b.p, x, r, scale, sfac, red, S_RES, st);
            ProfEnd();
            rr = ReadSlot(S_RES);
            restarts++;
        }
    }
    out->iters_outer = restarts;
    out->iters_inner = its;
    out->rel_res = bn2 > 0.0 ? std::sqrt(rr / bn2) : 0.0;
    *xOut = x;
    return status;
}

int Context::Solve(double tol, double **xOut, nb_result *out, const double *guess, double refNorm)
{
    if (!(tol > 0.0)) throw InputError("tolerance must be positive");
    if (n == 0)
    {
        xa.zero(st);
        *xOut = xa.p;
        out->b_norm = 0.0;
        out->rel_res = 0.0;
        out->iters_inner = out->iters_outer = 0;
        return NB_OK;
    }
    const int status = opt.precision == NB_PRECISION_MIXED ? SolveMixed(tol, xOut, out, guess, refNorm)
                                                           : SolveFP64(tol, xOut, out, guess, refNorm);
    solvesOnShape++;
    return status;
}

// ---------------------------------------------------------------------------------------------------------------
// the pressure step and projection
// ---------------------------------------------------------------------------------------------------------------
int Context::ProjectDevice(double *u, double *v, double *w, double *p, double rho, double dt, int compat, double tol,
                           nb_result *out, bool solve, bool correct, const double *pPrev, int scheme, bool warm)
{
    if (!built) throw InputError("set_layout has not been called");
    if (!u || !v || !p || (dim == 3 && !w)) throw InputError("null field pointer");
    if (!(rho > 0.0) || !(dt > 0.0)) throw InputError("rho and dt must be positive");
    if (scheme != NB_SCHEME_CHORIN && scheme != NB_SCHEME_INCREMENTAL) throw InputError("unknown scheme");
    const bool incr = scheme == NB_SCHEME_INCREMENTAL;
    if ((incr || warm) && !pPrev) throw InputError("the previous pressure is required");
    if (incr && !(solve && correct)) throw InputError("the incremental scheme runs the whole step");
    std::memset(out, 0, sizeof(*out));
    out->n = n;
    out->singular = singular ? 1 : 0;
    out->levels = (int)L.size();
    const LevelView v0 = L[0].view();
    NB_CK(cudaEventRecord(ev0, st));
    if (!solve)
    {
        ProfBegin(NB_K_PROJECT, (8.0 + 1.0 + 6.0 * 8.0) * (double)Cells());
        LaunchProject(v0, u, v, w, p, dt / rho, st);
        ProfEnd();
        LaunchMaxDiv(v0, u, v, w, dh, red, S_DIV, st);
        NB_CK(cudaEventRecord(ev1, st));
        NB_CK(cudaGetLastError());
        out->max_div = ReadSlot(S_DIV);
        float ms = 0.0f;
        NB_CK(cudaEventElapsedTime(&ms, ev0, ev1));
        out->seconds = ms * 1e-3;
        out->status = NB_OK;
        return NB_OK;
    }
    LaunchRing(v0, p, st); // EnforcePressureBC at the start of SolveScheme
    const double *pKnown = p; // the values DirichletSum reads on PRESSURE cells
    if (incr)
    {
        // SolveIncremental: the known Dirichlet values are p_b(t^{n+1}) - p_b(t^n); p_b(t^{n+1}) is kept for the end
        pSave.alloc(Cells());
        dq.alloc(Cells());
        NB_CK(cudaMemcpyAsync(pSave.p, p, pSave.bytes(), cudaMemcpyDeviceToDevice, st));
        LaunchCellwise(v0, CELL_DELTA, const_cast<double *>(p), pPrev, dq.p, st);
        pKnown = dq.p;
    }
    ProfBegin(NB_K_RHS, (3.0 * 8.0 + 1.0 + 8.0) * (double)Cells());
    LaunchRhs(v0, u, v, w, pKnown, rho / dt, scale, dh, b.p, st);
    ProfEnd();
    const bool compatOn = compat && singular && n > 0;
    if (compatOn)
        for (int pass = 0; pass < 2; pass++) // b -= mean(b), twice (PressureSolver3D.cpp:300-307)
        {
            LaunchSumUnknowns(v0, b.p, red, S_SUM, st);
            LaunchSubMeanScatter(v0, b.p, slots.p + S_SUM, n, 1, nullptr, st);
        }
    const double *guess = nullptr;
    double refNorm = 0.0;
    if (incr && n > 0)
    {
        // IncrementReferenceNorm: ||b + A p^n|| over the unknowns, the stopping floor of the increment's solve
        LaunchCellwise(v0, CELL_NEG, const_cast<double *>(pPrev), nullptr, xb.p, st);
        if (opt.precision == NB_PRECISION_MIXED)
            LaunchResidual64<float>(v0, b.p, xb.p, L[0].r32.p, scale, 1.0, red, S_RES, st);
        else
            LaunchResidual64<double>(v0, b.p, xb.p, L[0].r64.p, scale, 1.0, red, S_RES, st);
        refNorm = std::sqrt(ReadSlot(S_RES));
    }
    else if (warm && !nonuniform && n > 0)
    {
        // BuildWarmStartGuess: x0 = p^n on the unknowns, mean-free for a singular system with compatibility on
        LaunchCellwise(v0, CELL_TAKE, const_cast<double *>(pPrev), nullptr, xb.p, st);
        if (compatOn)
        {
            LaunchSumUnknowns(v0, xb.p, red, S_SUM, st);
            LaunchSubMeanScatter(v0, xb.p, slots.p + S_SUM, n, 1, nullptr, st);
        }
        guess = xb.p;
    }
    double *x = nullptr;
    const int status = Solve(tol, &x, out, guess, refNorm);
    // LevelPressure's mean removal (PressureSolver3D.cpp:181-187), then the scatter into p; the increment is not
    // levelled (its constant does not enter the gradient)
    const bool level = compatOn && !incr;
    if (level) LaunchSumUnknowns(v0, x, red, S_SUM, st);
    LaunchSubMeanScatter(v0, x, slots.p + S_SUM, n, level ? 1 : 0, p, st);
    LaunchRing(v0, p, st);
    if (incr) LaunchCellwise(v0, CELL_RING_DELTA, p, pPrev, nullptr, st); // the ring carries phi (:321-328)
    const bool toHost = hostP && !incr && correct;
    if (toHost)
    {
        // p is final: its copy to the host runs beside the velocity correction
        if (!cst) NB_CK(cudaStreamCreateWithFlags(&cst, cudaStreamNonBlocking));
        if (!evP) NB_CK(cudaEventCreateWithFlags(&evP, cudaEventDisableTiming));
        if (!evPDone) NB_CK(cudaEventCreateWithFlags(&evPDone, cudaEventDisableTiming));
        NB_CK(cudaEventRecord(evP, st));
        NB_CK(cudaStreamWaitEvent(cst, evP, 0));
        NB_CK(cudaMemcpyAsync(hostP, p, Cells() * sizeof(double), cudaMemcpyDeviceToHost, cst));
        hostCopied = true;
    }
    if (correct)
    {
        ProfBegin(NB_K_PROJECT, (8.0 + 1.0 + 6.0 * 8.0) * (double)Cells());
        LaunchProject(v0, u, v, w, p, dt / rho, st);
        ProfEnd();
        if (toHost)
        {
            // u, v, w are final: their copies follow p's, beside the divergence check
            NB_CK(cudaEventRecord(evP, st));
            NB_CK(cudaStreamWaitEvent(cst, evP, 0));
            NB_CK(cudaMemcpyAsync(hostU, u, FieldSizeU() * sizeof(double), cudaMemcpyDeviceToHost, cst));
            NB_CK(cudaMemcpyAsync(hostV, v, FieldSizeV() * sizeof(double), cudaMemcpyDeviceToHost, cst));
            if (dim == 3)
                NB_CK(cudaMemcpyAsync(hostW, w, FieldSizeW() * sizeof(double), cudaMemcpyDeviceToHost, cst));
            NB_CK(cudaEventRecord(evPDone, cst));
        }
        LaunchMaxDiv(v0, u, v, w, dh, red, S_DIV, st);
    }
    if (incr)
    {
        // AccumulatePressureIncrement (:374-393): p = p^n + phi on the unknowns, levelled, scattered, then
        // EnforcePressureBC with the prescribed values kept from the start
        double *acc = (x == xa.p) ? xb.p : xa.p;
        LaunchCellwise(v0, CELL_SUM, const_cast<double *>(pPrev), p, acc, st);
        if (compatOn) LaunchSumUnknowns(v0, acc, red, S_SUM, st);
        LaunchSubMeanScatter(v0, acc, slots.p + S_SUM, n, compatOn ? 1 : 0, p, st);
        LaunchCellwise(v0, CELL_RESTORE, p, pSave.p, nullptr, st);
        LaunchRing(v0, p, st);
    }
    NB_CK(cudaEventRecord(ev1, st));
    NB_CK(cudaGetLastError());
    out->max_div = correct ? ReadSlot(S_DIV) : -1.0;
    NB_CK(cudaEventSynchronize(ev1));
    float ms = 0.0f;
    NB_CK(cudaEventElapsedTime(&ms, ev0, ev1));
    out->seconds = ms * 1e-3;
    out->status = status;
    lastIterations = out->iters_inner;
    return status;
}

void Context::BatchBegin(double *u, double *v, double *w, double *p, double rho, double dt, int compat)
{
    if (!built) throw InputError("set_layout has not been called");
    if (!u || !v || !p || (dim == 3 && !w)) throw InputError("null field pointer");
    if (!(rho > 0.0) || !(dt > 0.0)) throw InputError("rho and dt must be positive");
    const LevelView v0 = L[0].view();
    LaunchRing(v0, p, st);
    LaunchRhs(v0, u, v, w, p, rho / dt, scale, dh, b.p, st);
    if (compat && singular && n > 0)
        for (int pass = 0; pass < 2; pass++) // b -= mean(b), twice (PressureSolver3D.cpp:300-307)
        {
            LaunchSumUnknowns(v0, b.p, red, S_SUM, st);
            LaunchSubMeanScatter(v0, b.p, slots.p + S_SUM, n, 1, nullptr, st);
        }
}

void Context::BatchEnd(double *x, double *u, double *v, double *w, double *p, double rho, double dt, int compat)
{
    const LevelView v0 = L[0].view();
    const bool level = compat && singular && n > 0;
    if (level) LaunchSumUnknowns(v0, x, red, S_SUM, st);
    LaunchSubMeanScatter(v0, x, slots.p + S_SUM, n, level ? 1 : 0, p, st);
    LaunchRing(v0, p, st);
    LaunchProject(v0, u, v, w, p, dt / rho, st);
    LaunchMaxDiv(v0, u, v, w, dh, red, S_DIV, st);
}

int Context::SolveLaplacian(const double *f, double *xh, double tol, nb_result *out)
{
    if (!built) throw InputError("set_layout has not been called");
    EnsureIdp();
    std::memset(out, 0, sizeof(*out));
    out->n = n;
    out->singular = singular ? 1 : 0;
    out->levels = (int)L.size();
    out->max_div = -1.0;
    if (n == 0) return NB_BAD_INPUT; // SolveLaplacian returns false on an empty system
    const LevelView v0 = L[0].view();
    DevArray<double> fc;
    fc.upload(f, (size_t)n, st);
    b.zero(st);
    LaunchScatterVolume(v0, idp.p, fc.p, b.p, 1, st); // b = f * CellVolume (PressureSolver3D.cpp:360-369)
    NB_CK(cudaEventRecord(ev0, st));
    double *x = nullptr;
    const int status = Solve(tol, &x, out);
    NB_CK(cudaEventRecord(ev1, st));
    LaunchGather(v0, idp.p, x, fc.p, st);
    NB_CK(cudaMemcpyAsync(xh, fc.p, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, st));
    NB_CK(cudaStreamSynchronize(st));
    float ms = 0.0f;
    NB_CK(cudaEventElapsedTime(&ms, ev0, ev1));
    out->seconds = ms * 1e-3;
    out->status = status;
    lastIterations = out->iters_inner;
    return status;
}

void Context::Rhs(const double *u, const double *v, const double *w, const double *p, double rho, double dt,
                  double *bOut)
{
    if (!built) throw InputError("set_layout has not been called");
    EnsureIdp();
    const LevelView v0 = L[0].view();
    DevArray<double> U, V, W, P, bc;
    U.upload(u, FieldSizeU(), st);
    V.upload(v, FieldSizeV(), st);
    if (dim == 3) W.upload(w, FieldSizeW(), st);
    P.upload(p, Cells(), st);
    LaunchRing(v0, P.p, st);
    b.zero(st);
    LaunchRhs(v0, U.p, V.p, W.p, P.p, rho / dt, scale, dh, b.p, st);
    bc.alloc((size_t)std::max(n, 1));
    LaunchGather(v0, idp.p, b.p, bc.p, st);
    if (n) NB_CK(cudaMemcpyAsync(bOut, bc.p, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, st));
    NB_CK(cudaStreamSynchronize(st));
}

void Context::ExportMatrix(int32_t *rowptr, int32_t *col, double *val, int *nnzOut, int *singularOut)
{
    if (!built) throw InputError("set_layout has not been called");
    EnsureIdp();
    const LevelView v0 = L[0].view();
    const size_t cap = (size_t)std::max(n, 1) * (dim == 3 ? 7 : 5);
    DevArray<int> rowLen, rowPtr, flag;
    DevArray<int32_t> c;
    DevArray<double> vv;
    rowLen.alloc((size_t)n + 1);
    rowPtr.alloc((size_t)n + 1);
    flag.alloc(1);
    c.alloc(cap);
    vv.alloc(cap);
    int nnz = 0, sing = 0;
    nb::ExportMatrix(v0, idp.p, n, scale, rowLen.p, rowPtr.p, c.p, vv.p, flag.p, scanTmp.p, scanTmpBytes, &nnz, &sing,
                     st);
    NB_CK(cudaMemcpyAsync(rowptr, rowPtr.p, sizeof(int) * ((size_t)n + 1), cudaMemcpyDeviceToHost, st));
    if (nnz)
    {
        NB_CK(cudaMemcpyAsync(col, c.p, sizeof(int32_t) * (size_t)nnz, cudaMemcpyDeviceToHost, st));
        NB_CK(cudaMemcpyAsync(val, vv.p, sizeof(double) * (size_t)nnz, cudaMemcpyDeviceToHost, st));
    }
    NB_CK(cudaStreamSynchronize(st));
    *nnzOut = nnz;
    *singularOut = sing;
}

void Context::EnsureIdp()
{
    if (idpValid) return;
    ArrayPoolScope pooled(&arrays);
    const LevelView v0 = L[0].view();
    idp.alloc(Cells());
    lineCounts.alloc((size_t)std::max(v0.nLines, 0) + 1);
    lineOffsets.alloc((size_t)std::max(v0.nLines, 0) + 1);
    lineCounts.zero(st);
    size_t need = std::max(ScanTempBytes(std::max(v0.nLines, 0) + 1), ScanTempBytes(1 << 20));
    if (need > scanTmpBytes)
    {
        scanTmp.alloc(need);
        scanTmpBytes = need;
    }
    int total = 0;
    NumberUnknowns(v0, idp.p, lineCounts.p, lineOffsets.p, scanTmp.p, scanTmpBytes, &total, st);
    if (total != n) throw CudaError("IDP numbering disagrees with the unknown count", cudaErrorUnknown);
    idpValid = true;
}

void Context::GetIdp(int32_t *out)
{
    if (!built) throw InputError("set_layout has not been called");
    EnsureIdp();
    NB_CK(cudaMemcpyAsync(out, idp.p, sizeof(int32_t) * Cells(), cudaMemcpyDeviceToHost, st));
    NB_CK(cudaStreamSynchronize(st));
}

template void Context::VCycle<float>(int, float *, float *);
template void Context::VCycle<double>(int, double *, double *);

} // namespace nb
