// The extern "C" entry points of include/nereus_b200.h. Every call catches its own exceptions and turns them into an
// nb_status; the message of the last failure on this host thread is kept for nereus_b200_last_error().
#include "nb_guard.h"

#include <memory>
#include <new>
#include <string>

struct nb_ctx
{
    std::unique_ptr<nb::Context> c;
};

namespace nb
{
namespace capi
{
thread_local std::string g_error;
}
} // namespace nb
using nb::capi::Fail;
using nb::capi::Guard;
using nb::capi::g_error;

extern "C" {

void nereus_b200_default_options(nb_options *o)
{
    if (!o) return;
    o->device = 0;
    o->precision = NB_PRECISION_MIXED;
    o->max_iters = 60;
    o->max_outer = 12;
    o->inner_tol = 1e-4;
    o->pre_sweeps = 1;
    o->post_sweeps = 1;
    o->coarse_sweeps = 4;
    o->max_levels = 16;
    o->stream = nullptr;
    o->use_graphs = 2;
    o->transfer_kernels = 0;
    o->pair_kernels = 2;
    o->tail_cells = 2048;
    o->stretched_sweeps = 2;
    o->autotune = 1;
    o->skip_idle_tiles = 1;
    o->x_groups = 1;
}

const char *nereus_b200_last_error(void) { return g_error.c_str(); }

int nereus_b200_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

int nereus_b200_create(nb_ctx **ctx, const nb_options *opt)
{
    if (!ctx) return Fail(NB_BAD_INPUT, "ctx is null");
    *ctx = nullptr;
    return Guard([&] {
        nb_options o;
        nereus_b200_default_options(&o);
        if (opt) o = *opt;
        if (o.precision != NB_PRECISION_FP64 && o.precision != NB_PRECISION_MIXED)
            throw nb::InputError("unknown precision");
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
            return Fail(NB_NO_DEVICE, "no CUDA device");
        if (o.device < 0 || o.device >= count) throw nb::InputError("device ordinal out of range");
        auto *h = new nb_ctx;
        try
        {
            h->c.reset(new nb::Context(o));
        }
        catch (...)
        {
            delete h;
            throw;
        }
        *ctx = h;
        return (int)NB_OK;
    });
}

void nereus_b200_destroy(nb_ctx *ctx)
{
    if (!ctx) return;
    try
    {
        if (ctx->c) cudaSetDevice(ctx->c->device);
        ctx->c.reset();
    }
    catch (...)
    {
    }
    delete ctx;
}

int nereus_b200_set_layout(nb_ctx *ctx, int dim, int Nx, int Ny, int Nz, const uint8_t *cellTypes,
                           const double *const width[3], const double *const gap[3], int nonUniform, double dh)
{
    if (!ctx || !ctx->c) return Fail(NB_BAD_INPUT, "ctx is null");
    return Guard([&] {
        NB_CK(cudaSetDevice(ctx->c->device));
        ctx->c->SetLayout(dim, Nx, Ny, Nz, cellTypes, width, gap, nonUniform, dh);
        return (int)NB_OK;
    });
}

int nereus_b200_project(nb_ctx *ctx, double *u, double *v, double *w, double *p, double rho, double dt, int scheme,
                        int needsCompat, double tol, nb_result *out)
{
    if (!ctx || !ctx->c) return Fail(NB_BAD_INPUT, "ctx is null");
    if (scheme != NB_SCHEME_CHORIN) return Fail(NB_BAD_INPUT, "only the Chorin scheme is served");
    return Guard([&] {
        nb::Context &C = *ctx->c;
        NB_CK(cudaSetDevice(C.device));
        if (!C.built) throw nb::InputError("set_layout has not been called");
        if (!u || !v || !p || (C.dim == 3 && !w)) throw nb::InputError("null field pointer");
        nb_result local{};
        nb_result *r = out ? out : &local;
        C.du.upload(u, C.FieldSizeU(), C.st);
        C.dv.upload(v, C.FieldSizeV(), C.st);
        if (C.dim == 3) C.dw.upload(w, C.FieldSizeW(), C.st);
        C.dp.upload(p, C.Cells(), C.st);
        // p and then u, v, w go back to the host on the context's copy stream as soon as each is final, beside the
        // velocity correction and the divergence check
        struct HostFields
        {
            nb::Context &C;
            HostFields(nb::Context &c, double *u, double *v, double *w, double *p) : C(c)
            {
                C.hostU = u;
                C.hostV = v;
                C.hostW = w;
                C.hostP = p;
                C.hostCopied = false;
            }
            ~HostFields()
            {
                if (C.hostCopied) cudaStreamSynchronize(C.cst); // an error path must not leave the copies running
                C.hostP = C.hostU = C.hostV = C.hostW = nullptr;
            }
        } hf(C, u, v, w, p);
        const int status = C.ProjectDevice(C.du.p, C.dv.p, C.dim == 3 ? C.dw.p : C.du.p, C.dp.p, rho, dt,
                                           needsCompat, tol, r);
        if (C.hostCopied)
            NB_CK(cudaStreamWaitEvent(C.st, C.evPDone, 0));
        else
        {
            NB_CK(cudaMemcpyAsync(u, C.du.p, C.du.bytes(), cudaMemcpyDeviceToHost, C.st));
            NB_CK(cudaMemcpyAsync(v, C.dv.p, C.dv.bytes(), cudaMemcpyDeviceToHost, C.st));
            if (C.dim == 3) NB_CK(cudaMemcpyAsync(w, C.dw.p, C.dw.bytes(), cudaMemcpyDeviceToHost, C.st));
            NB_CK(cudaMemcpyAsync(p, C.dp.p, C.dp.bytes(), cudaMemcpyDeviceToHost, C.st));
        }
        NB_CK(cudaStreamSynchronize(C.st));
        return status;
    });
}

int nereus_b200_project_ex(nb_ctx *ctx, double *u, double *v, double *w, double *p, const double *pPrev, double rho,
                           double dt, int scheme, int needsCompat, int warmStart, double tol, nb_result *out)
{
    if (!ctx || !ctx->c) return Fail(NB_BAD_INPUT, "ctx is null");
    return Guard([&] {
        nb::Context &C = *ctx->c;
        NB_CK(cudaSetDevice(C.device));
        if (!C.built) throw nb::InputError("set_layout has not been called");
        if (!u || !v || !p || (C.dim == 3 && !w)) throw nb::InputError("null field pointer");
        nb_result local{};
        nb_result *r = out ? out : &local;
        C.du.upload(u, C.FieldSizeU(), C.st);
        C.dv.upload(v, C.FieldSizeV(), C.st);
        if (C.dim == 3) C.dw.upload(w, C.FieldSizeW(), C.st);
        C.dp.upload(p, C.Cells(), C.st);
        if (pPrev) C.dpPrev.upload(pPrev, C.Cells(), C.st);
        const int status = C.ProjectDevice(C.du.p, C.dv.p, C.dim == 3 ? C.dw.p : C.du.p, C.dp.p, rho, dt,
                                           needsCompat, tol, r, true, true, pPrev ? C.dpPrev.p : nullptr, scheme,
                                           warmStart != 0);
        NB_CK(cudaMemcpyAsync(u, C.du.p, C.du.bytes(), cudaMemcpyDeviceToHost, C.st));
        NB_CK(cudaMemcpyAsync(v, C.dv.p, C.dv.bytes(), cudaMemcpyDeviceToHost, C.st));
        if (C.dim == 3) NB_CK(cudaMemcpyAsync(w, C.dw.p, C.dw.bytes(), cudaMemcpyDeviceToHost, C.st));
        NB_CK(cudaMemcpyAsync(p, C.dp.p, C.dp.bytes(), cudaMemcpyDeviceToHost, C.st));
        NB_CK(cudaStreamSynchronize(C.st));
        return status;
    });
}

int nereus_b200_project_device_ex(nb_ctx *ctx, double *d_u, double *d_v, double *d_w, double *d_p,
                                  const double *d_pPrev, double rho, double dt, int scheme, int needsCompat,
                                  int warmStart, double tol, nb_result *out)
{
    if (!ctx || !ctx->c) return Fail(NB_BAD_INPUT, "ctx is null");
    return Guard([&] {
        nb::Context &C = *ctx->c;
        NB_CK(cudaSetDevice(C.device));
        nb_result local{};
        return C.ProjectDevice(d_u, d_v, C.dim == 3 ? d_w : d_u, d_p, rho, dt, needsCompat, tol, out ? out : &local,
                               true, true, d_pPrev, scheme, warmStart != 0);
    });
}

int nereus_b200_solve_pressure(nb_ctx *ctx, const double *u, const double *v, const double *w, double *p, double rho,
                               double dt, int scheme, int needsCompat, double tol, nb_result *out)
{
    if (!ctx || !ctx->c) return Fail(NB_BAD_INPUT, "ctx is null");
    if (scheme != NB_SCHEME_CHORIN) return Fail(NB_BAD_INPUT, "only the Chorin scheme is served");
    return Guard([&] {
        nb::Context &C = *ctx->c;
        NB_CK(cudaSetDevice(C.device));
        if (!C.built) throw nb::InputError("set_layout has not been called");
        if (!u || !v || !p || (C.dim == 3 && !w)) throw nb::InputError("null field pointer");
        nb_result local{};
        C.du.upload(u, C.FieldSizeU(), C.st);
        C.dv.upload(v, C.FieldSizeV(), C.st);
        if (C.dim == 3) C.dw.upload(w, C.FieldSizeW(), C.st);
        C.dp.upload(p, C.Cells(), C.st);
        const int status = C.ProjectDevice(C.du.p, C.dv.p, C.dim == 3 ? C.dw.p : C.du.p, C.dp.p, rho, dt,
                                           needsCompat, tol, out ? out : &local, true, false);
        NB_CK(cudaMemcpyAsync(p, C.dp.p, C.dp.bytes(), cudaMemcpyDeviceToHost, C.st));
        NB_CK(cudaStreamSynchronize(C.st));
        return status;
    });
}

int nereus_b200_project_velocity(nb_ctx *ctx, double *u, double *v, double *w, const double *p, double rho,
                                 double dt)
{
    if (!ctx || !ctx->c) return Fail(NB_BAD_INPUT, "ctx is null");
    return Guard([&] {
        nb::Context &C = *ctx->c;
        NB_CK(cudaSetDevice(C.device));
        if (!C.built) throw nb::InputError("set_layout has not been called");
        if (!u || !v || !p || (C.dim == 3 && !w)) throw nb::InputError("null field pointer");
        nb_result local{};
        C.du.upload(u, C.FieldSizeU(), C.st);
        C.dv.upload(v, C.FieldSizeV(), C.st);
        if (C.dim == 3) C.dw.upload(w, C.FieldSizeW(), C.st);
        C.dp.upload(p, C.Cells(), C.st);
        C.ProjectDevice(C.du.p, C.dv.p, C.dim == 3 ? C.dw.p : C.du.p, C.dp.p, rho, dt, 0, 1.0, &local, false, true);
        NB_CK(cudaMemcpyAsync(u, C.du.p, C.du.bytes(), cudaMemcpyDeviceToHost, C.st));
        NB_CK(cudaMemcpyAsync(v, C.dv.p, C.dv.bytes(), cudaMemcpyDeviceToHost, C.st));
        if (C.dim == 3) NB_CK(cudaMemcpyAsync(w, C.dw.p, C.dw.bytes(), cudaMemcpyDeviceToHost, C.st));
        NB_CK(cudaStreamSynchronize(C.st));
        return (int)NB_OK;
    });
}

int nereus_b200_project_device(nb_ctx *ctx, double *d_u, double *d_v, double *d_w, double *d_p, double rho,
                               double dt, int needsCompat, double tol, nb_result *out)
{
    if (!ctx || !ctx->c) return Fail(NB_BAD_INPUT, "ctx is null");
    return Guard([&] {
        nb::Context &C = *ctx->c;
        NB_CK(cudaSetDevice(C.device));
        nb_result local{};
        return C.ProjectDevice(d_u, d_v, C.dim == 3 ? d_w : d_u, d_p, rho, dt, needsCompat, tol, out ? out : &local);
    });
}

int nereus_b200_solve_laplacian(nb_ctx *ctx, const double *f, double *x, double tol, nb_result *out)
{
    if (!ctx || !ctx->c) return Fail(NB_BAD_INPUT, "ctx is null");
    if (!f || !x) return Fail(NB_BAD_INPUT, "null vector");
    return Guard([&] {
        nb::Context &C = *ctx->c;
        NB_CK(cudaSetDevice(C.device));
        nb_result local{};
        return C.SolveLaplacian(f, x, tol, out ? out : &local);
    });
}

int nereus_b200_system_size(const nb_ctx *ctx) { return ctx && ctx->c && ctx->c->built ? ctx->c->n : 0; }

int nereus_b200_last_iterations(const nb_ctx *ctx) { return ctx && ctx->c ? ctx->c->lastIterations : 0; }

int nereus_b200_get_idp(nb_ctx *ctx, int32_t *idp)
{
    if (!ctx || !ctx->c || !idp) return Fail(NB_BAD_INPUT, "null argument");
    return Guard([&] {
        NB_CK(cudaSetDevice(ctx->c->device));
        ctx->c->GetIdp(idp);
        return (int)NB_OK;
    });
}

int nereus_b200_number_unknowns_noalloc(int device, int dim, int Nx, int Ny, int Nz, const uint8_t *cellTypes,
                                        int32_t *idp, int32_t *n, void *stream)
{
    static_assert(NB_NOALLOC_MAX_LINES == nb::kNoAllocMaxLines, "header and library disagree on the limit");
    return Guard([&] {
        int count = 0;
        NB_CK(cudaGetDeviceCount(&count));
        if (device < 0 || device >= count) throw nb::InputError("no such device");
        int prev = 0;
        NB_CK(cudaGetDevice(&prev));
        NB_CK(cudaSetDevice(device));
        try
        {
            nb::NumberUnknownsNoAlloc(device, dim, Nx, Ny, Nz, cellTypes, idp, n, (cudaStream_t)stream);
        }
        catch (...)
        {
            cudaSetDevice(prev);
            throw;
        }
        NB_CK(cudaSetDevice(prev));
        return (int)NB_OK;
    });
}

} // extern "C"

struct nb_bc
{
    nb::BcReplay *r = nullptr;
    ~nb_bc() { nb::DestroyBcReplay(r); }
};

namespace
{
// Runs f with `device` current, restoring the caller's device afterwards.
template <typename F> void OnDevice(int device, F &&f)
{
    int prev = 0;
    NB_CK(cudaGetDevice(&prev));
    NB_CK(cudaSetDevice(device));
    try
    {
        f();
    }
    catch (...)
    {
        cudaSetDevice(prev);
        throw;
    }
    NB_CK(cudaSetDevice(prev));
}
} // namespace

extern "C" {

int nereus_b200_bc_create(int device, const nb_bc_lists *lists, nb_bc **out)
{
    if (!lists || !out) return Fail(NB_BAD_INPUT, "null argument");
    *out = nullptr;
    return Guard([&] {
        nb::CheckBcLists(*lists); // bad lists fail here, before any device
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return Fail(NB_NO_DEVICE, "no CUDA device");
        if (device < 0 || device >= ndev) throw nb::InputError("no such device");
        std::unique_ptr<nb_bc> b(new nb_bc);
        OnDevice(device, [&] { b->r = nb::CreateBcReplay(device, *lists); });
        *out = b.release();
        return (int)NB_OK;
    });
}

int nereus_b200_bc_enforce_velocity(nb_bc *bc, double *u, double *v, double *w, const double *presc_values,
                                    void *stream)
{
    if (!bc || !bc->r) return Fail(NB_BAD_INPUT, "null argument");
    return Guard([&] {
        OnDevice(nb::BcDevice(*bc->r), [&] {
            nb::EnforceVelocityDevice(*bc->r, u, v, w, presc_values, (cudaStream_t)stream);
        });
        return (int)NB_OK;
    });
}

int nereus_b200_bc_enforce_pressure(nb_bc *bc, double *p, const double *ring_values, void *stream)
{
    if (!bc || !bc->r) return Fail(NB_BAD_INPUT, "null argument");
    return Guard([&] {
        OnDevice(nb::BcDevice(*bc->r), [&] { nb::EnforcePressureDevice(*bc->r, p, ring_values, (cudaStream_t)stream); });
        return (int)NB_OK;
    });
}

int nereus_b200_bc_plan(const nb_bc_lists *lists, int32_t *velocity_level, int32_t *pressure_level,
                        int *velocity_levels, int *pressure_levels)
{
    if (!lists) return Fail(NB_BAD_INPUT, "null argument");
    return Guard([&] {
        std::vector<int> vel, pres;
        nb::PlanBcLevels(*lists, vel, pres);
        int nv = 0, np = 0;
        for (size_t q = 0; q < vel.size(); q++)
        {
            if (velocity_level) velocity_level[q] = vel[q];
            if (vel[q] + 1 > nv) nv = vel[q] + 1;
        }
        for (size_t q = 0; q < pres.size(); q++)
        {
            if (pressure_level) pressure_level[q] = pres[q];
            if (pres[q] + 1 > np) np = pres[q] + 1;
        }
        if (velocity_levels) *velocity_levels = nv;
        if (pressure_levels) *pressure_levels = np;
        return (int)NB_OK;
    });
}

int nereus_b200_bc_levels(const nb_bc *bc, int *velocity_levels, int *pressure_levels)
{
    if (!bc || !bc->r) return Fail(NB_BAD_INPUT, "null argument");
    if (velocity_levels) *velocity_levels = nb::BcLevels(*bc->r, 0);
    if (pressure_levels) *pressure_levels = nb::BcLevels(*bc->r, 1);
    return NB_OK;
}

void nereus_b200_bc_destroy(nb_bc *bc)
{
    if (!bc) return;
    int prev = 0;
    const bool ok = cudaGetDevice(&prev) == cudaSuccess;
    if (bc->r) cudaSetDevice(nb::BcDevice(*bc->r));
    delete bc;
    if (ok) cudaSetDevice(prev);
}

size_t nereus_b200_update_fluid_cells_scratch_bytes(int dim, int Nx, int Ny, int Nz)
{
    return nb::RelabelScratchBytes(dim, Nx, Ny, Nz);
}

int nereus_b200_update_fluid_cells_device(int device, int dim, int Nx, int Ny, int Nz, double ox, double oy,
                                          double oz, double dh, const double *px, const double *py, const double *pz,
                                          int64_t count, int64_t stride, uint8_t *cellTypes, void *scratch,
                                          size_t scratch_bytes, int64_t *skipped, void *stream)
{
    static_assert(sizeof(int64_t) == sizeof(unsigned long long), "skipped is a 64-bit counter");
    return Guard([&] {
        int ndev = 0;
        NB_CK(cudaGetDeviceCount(&ndev));
        if (device < 0 || device >= ndev) throw nb::InputError("no such device");
        int prev = 0;
        NB_CK(cudaGetDevice(&prev));
        NB_CK(cudaSetDevice(device));
        try
        {
            nb::UpdateFluidCellsDevice(dim, Nx, Ny, Nz, ox, oy, oz, dh, px, py, pz, count, stride, cellTypes, scratch,
                                       scratch_bytes, (unsigned long long *)skipped, (cudaStream_t)stream);
        }
        catch (...)
        {
            cudaSetDevice(prev);
            throw;
        }
        NB_CK(cudaSetDevice(prev));
        return (int)NB_OK;
    });
}

int nereus_b200_update_fluid_cells(int dim, int Nx, int Ny, int Nz, double ox, double oy, double oz, double dh,
                                   const double *px, const double *py, const double *pz, int64_t count,
                                   int64_t stride, uint8_t *cellTypes, int64_t *skipped)
{
    if (!cellTypes) return Fail(NB_BAD_INPUT, "null argument");
    if ((dim != 2 && dim != 3) || Nx < 1 || Ny < 1 || (dim == 3 && Nz < 1)) return Fail(NB_BAD_INPUT, "bad sizes");
    if (count < 0) return Fail(NB_BAD_INPUT, "negative particle count");
    if (count > 0 && (!px || !py || (dim == 3 && !pz))) return Fail(NB_BAD_INPUT, "null particle coordinates");
    if (count > 0 && stride < 1) return Fail(NB_BAD_INPUT, "particle stride must be at least 1");
    return Guard([&] {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return Fail(NB_NO_DEVICE, "no CUDA device");
        const int nz = dim == 3 ? Nz : 1;
        const size_t cells = (size_t)Nx * Ny * nz;
        // the positions packed as three plain arrays: 24 bytes per particle cross PCIe instead of the whole struct
        std::vector<double> xyz((size_t)count * (dim == 3 ? 3 : 2));
        double *hx = xyz.data(), *hy = hx + count, *hz = dim == 3 ? hy + count : nullptr;
        for (int64_t p = 0; p < count; p++)
        {
            hx[p] = px[p * stride];
            hy[p] = py[p * stride];
            if (hz) hz[p] = pz[p * stride];
        }
        cudaStream_t st;
        NB_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamDestroy(s); } } sg{st};
        nb::DevArray<double> P;
        nb::DevArray<uint8_t> T, S;
        nb::DevArray<unsigned long long> K;
        P.upload(xyz.data(), xyz.size(), st);
        T.upload(cellTypes, cells, st);
        const size_t sb = nb::RelabelScratchBytes(dim, Nx, Ny, Nz);
        S.alloc(sb);
        K.alloc(1);
        const double *dx = P.p, *dy = P.p ? P.p + count : nullptr, *dz = (P.p && dim == 3) ? P.p + 2 * count : nullptr;
        nb::UpdateFluidCellsDevice(dim, Nx, Ny, Nz, ox, oy, oz, dh, dx, dy, dz, count, 1, T.p, S.p, sb, K.p, st);
        unsigned long long k = 0;
        NB_CK(cudaMemcpyAsync(cellTypes, T.p, cells, cudaMemcpyDeviceToHost, st));
        NB_CK(cudaMemcpyAsync(&k, K.p, sizeof(k), cudaMemcpyDeviceToHost, st));
        NB_CK(cudaStreamSynchronize(st));
        if (skipped) *skipped = (int64_t)k;
        return (int)NB_OK;
    });
}

int nereus_b200_export_matrix(nb_ctx *ctx, int32_t *rowptr, int32_t *col, double *val, int *nnz, int *singular)
{
    if (!ctx || !ctx->c || !rowptr || !col || !val || !nnz || !singular) return Fail(NB_BAD_INPUT, "null argument");
    return Guard([&] {
        NB_CK(cudaSetDevice(ctx->c->device));
        ctx->c->ExportMatrix(rowptr, col, val, nnz, singular);
        return (int)NB_OK;
    });
}

int nereus_b200_rhs(nb_ctx *ctx, const double *u, const double *v, const double *w, const double *p, double rho,
                    double dt, double *b)
{
    if (!ctx || !ctx->c || !u || !v || !p || !b) return Fail(NB_BAD_INPUT, "null argument");
    return Guard([&] {
        nb::Context &C = *ctx->c;
        NB_CK(cudaSetDevice(C.device));
        if (C.dim == 3 && !w) throw nb::InputError("null w");
        C.Rhs(u, v, w, p, rho, dt, b);
        return (int)NB_OK;
    });
}

int nereus_b200_profile_enable(nb_ctx *ctx, unsigned kernelMask)
{
    if (!ctx || !ctx->c) return Fail(NB_BAD_INPUT, "ctx is null");
    return Guard([&] {
        NB_CK(cudaSetDevice(ctx->c->device));
        NB_CK(cudaStreamSynchronize(ctx->c->st));
        ctx->c->ProfClear();
        ctx->c->profMask = kernelMask;
        return (int)NB_OK;
    });
}

int nereus_b200_profile_read(nb_ctx *ctx, int kernelId, int *launches, double *totalMs, double *bytesPerLaunch)
{
    if (!ctx || !ctx->c || !launches || !totalMs || !bytesPerLaunch) return Fail(NB_BAD_INPUT, "null argument");
    if (kernelId < 0 || kernelId >= NB_K_COUNT) return Fail(NB_BAD_INPUT, "kernel id out of range");
    return Guard([&] {
        NB_CK(cudaSetDevice(ctx->c->device));
        ctx->c->ProfRead(kernelId, launches, totalMs, bytesPerLaunch);
        return (int)NB_OK;
    });
}

long long nereus_b200_kernel_launches(void) { return nb::g_launches.load(); }

int nereus_b200_label_cells(int dim, int Nx, int Ny, int Nz, const double *cx, const double *cy, const double *cz,
                            const nb_scene *scene, uint8_t *cellTypes)
{
    if (!cx || !cy || !cz || !scene || !cellTypes) return Fail(NB_BAD_INPUT, "null argument");
    if ((dim != 2 && dim != 3) || Nx < 1 || Ny < 1 || Nz < 1) return Fail(NB_BAD_INPUT, "bad sizes");
    if (scene->nregions < 0 || scene->nregions > 16) return Fail(NB_BAD_INPUT, "at most 16 regions");
    return Guard([&] {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return Fail(NB_NO_DEVICE, "no CUDA device");
        const int nz = dim == 3 ? Nz : 1;
        const size_t cells = (size_t)Nx * Ny * nz;
        cudaStream_t st;
        NB_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        nb::DevArray<double> X, Y, Z;
        nb::DevArray<uint8_t> T;
        X.upload(cx, (size_t)Nx, st);
        Y.upload(cy, (size_t)Ny, st);
        Z.upload(cz, (size_t)nz, st);
        T.alloc(cells);
        nb::LaunchLabelCells(dim, Nx, Ny, nz, X.p, Y.p, Z.p, *scene, T.p, st);
        NB_CK(cudaGetLastError());
        NB_CK(cudaMemcpyAsync(cellTypes, T.p, cells, cudaMemcpyDeviceToHost, st));
        NB_CK(cudaStreamSynchronize(st));
        cudaStreamDestroy(st);
        return (int)NB_OK;
    });
}

int nereus_b200_x_groups(const double *widths, int n, double yz_min, int32_t *counts)
{
    if (!widths || !counts || n < 1 || !(yz_min > 0.0)) return Fail(NB_BAD_INPUT, "bad x widths");
    std::vector<int> c;
    nb::PlanXGroups(widths, n, yz_min, c);
    for (size_t g = 0; g < c.size(); g++) counts[g] = c[g];
    return (int)c.size();
}

int nereus_b200_x_maps(const double *widths, int n, double yz_min, int32_t *xp, int32_t *xr)
{
    if (!widths || !xp || !xr || n < 1 || !(yz_min > 0.0)) return Fail(NB_BAD_INPUT, "bad x widths");
    int Nc = 0;
    std::vector<double> size;
    std::vector<int> p, r;
    if (!nb::XMaps(widths, n, yz_min, Nc, size, p, r)) return 0;
    for (size_t q = 0; q < p.size(); q++) xp[q] = p[q];
    for (size_t q = 0; q < r.size(); q++) xr[q] = r[q];
    return Nc;
}

} // extern "C"
