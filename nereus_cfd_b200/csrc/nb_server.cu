// Batched and served pressure steps: a queue of independent requests, run by slots (a host thread, a solver
// context and its CUDA stream) on one or more devices, with admission by a per-device memory budget.
//
// A request's layout (cell types, spacing tables) is copied at submission; its fields are read when a slot starts
// it and rewritten when it completes. A slot keeps its context between requests, so a run of requests with the same
// layout builds the multigrid hierarchy once (the context compares the layout bytes, as PressureLayoutChanged), and
// requests of equal size reuse its device buffers.
#include "nb_guard.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace nb
{
namespace
{

using Clock = std::chrono::steady_clock;

struct Request
{
    uint64_t ticket = 0;
    nb_request r{};
    std::vector<uint8_t> types;
    std::vector<double> tables[6]; // width x, y, z then gap x, y, z
    double bytes = 0.0;
    Clock::time_point submitted;
};

struct Record
{
    int state = 0; // 0 queued, 1 running, 2 done
    int status = NB_BUSY;
    nb_result result{};
    std::string error;
};

} // namespace

double RequestBytes(int dim, int Nx, int Ny, int Nz, int precision)
{
    const double cells = (double)Nx * Ny * (dim == 3 ? Nz : 1);
    // fields u, v, w, p, p_prev (5 x 8), b and two solutions (3 x 8), types/codes/du/pext (4), level-0 solver
    // vectors (r, e, res, p0, p1, q, x: 7 x 4 or 8) and the coarser levels (x 8/7 in 3D)
    const double s = precision == NB_PRECISION_MIXED ? 4.0 : 8.0;
    return cells * (5 * 8 + 3 * 8 + 4 + 7 * s * (dim == 3 ? 8.0 / 7.0 : 4.0 / 3.0)) + (64 << 20);
}

void Plan(const double *costs, int n, int k, int *deviceOf)
{
    std::vector<double> load((size_t)k, 0.0);
    for (int q = 0; q < n; q++)
    {
        int best = 0;
        for (int d = 1; d < k; d++)
            if (load[(size_t)d] < load[(size_t)best]) best = d;
        deviceOf[q] = best;
        load[(size_t)best] += costs[q];
    }
}

} // namespace nb

struct nb_server
{
    nb_server_options opt{};
    std::vector<int> devices;
    std::mutex mu;
    std::condition_variable cv;      // work for the slots, completions for the waiters
    std::deque<std::unique_ptr<nb::Request>> queue;
    std::unordered_map<uint64_t, nb::Record> records;
    std::vector<double> used;        // admitted bytes per device
    std::vector<long long> doneOn;   // completions per device
    std::vector<double> latencies;   // ms
    double layoutSeconds = 0.0, projectSeconds = 0.0; // slots' host time in set_layout and in the step
    long long submitted = 0, completed = 0, failed = 0, running = 0;
    uint64_t nextTicket = 1;
    bool started = false, stop = false;
    nb::Clock::time_point first;
    double budget = 0.0;
    std::vector<std::thread> slots;

    void Slot(int dev);
    bool Fits(const nb::Request &q, int dev) const { return used[(size_t)dev] + q.bytes <= budget; }
};

void nb_server::Slot(int dev)
{
    if (cudaSetDevice(devices[(size_t)dev]) != cudaSuccess) return;
    std::unique_ptr<nb::Context> ctx;
    for (;;)
    {
        std::unique_ptr<nb::Request> q;
        {
            std::unique_lock<std::mutex> lock(mu);
            for (;;)
            {
                if (stop) return;
                auto it = std::find_if(queue.begin(), queue.end(),
                                       [&](const std::unique_ptr<nb::Request> &x) { return Fits(*x, dev); });
                if (it != queue.end())
                {
                    q = std::move(*it);
                    queue.erase(it);
                    break;
                }
                cv.wait(lock);
            }
            used[(size_t)dev] += q->bytes;
            running++;
            records[q->ticket].state = 1;
        }
        nb_result res{};
        int status = NB_OK;
        std::string err;
        double tLayout = 0.0, tProject = 0.0;
        try
        {
            if (!ctx)
            {
                nb_options o = opt.solver;
                o.device = devices[(size_t)dev];
                o.stream = nullptr;
                ctx = std::make_unique<nb::Context>(o);
            }
            nb::Context &C = *ctx;
            const nb_request &r = q->r;
            const double *W[3] = {q->tables[0].data(), q->tables[1].data(), q->tables[2].data()};
            const double *G[3] = {q->tables[3].data(), q->tables[4].data(), q->tables[5].data()};
            const auto t0 = nb::Clock::now();
            C.SetLayout(r.dim, r.Nx, r.Ny, r.Nz, q->types.data(), W, G, r.non_uniform, r.dh);
            tLayout = std::chrono::duration<double>(nb::Clock::now() - t0).count();
            if (r.fields_on_device)
            {
                // the caller's device fields, in place
                status = C.ProjectDevice(r.u, r.v, C.dim == 3 ? r.w : r.u, r.p, r.rho, r.dt, r.needs_compat, r.tol,
                                         &res, true, true, r.p_prev, r.scheme, r.warm_start != 0);
            }
            else
            {
                C.du.upload(r.u, C.FieldSizeU(), C.st);
                C.dv.upload(r.v, C.FieldSizeV(), C.st);
                if (C.dim == 3) C.dw.upload(r.w, C.FieldSizeW(), C.st);
                C.dp.upload(r.p, C.Cells(), C.st);
                if (r.p_prev) C.dpPrev.upload(r.p_prev, C.Cells(), C.st);
                status = C.ProjectDevice(C.du.p, C.dv.p, C.dim == 3 ? C.dw.p : C.du.p, C.dp.p, r.rho, r.dt,
                                         r.needs_compat, r.tol, &res, true, true, r.p_prev ? C.dpPrev.p : nullptr,
                                         r.scheme, r.warm_start != 0);
                NB_CK(cudaMemcpyAsync(r.u, C.du.p, C.du.bytes(), cudaMemcpyDeviceToHost, C.st));
                NB_CK(cudaMemcpyAsync(r.v, C.dv.p, C.dv.bytes(), cudaMemcpyDeviceToHost, C.st));
                if (C.dim == 3) NB_CK(cudaMemcpyAsync(r.w, C.dw.p, C.dw.bytes(), cudaMemcpyDeviceToHost, C.st));
                NB_CK(cudaMemcpyAsync(r.p, C.dp.p, C.dp.bytes(), cudaMemcpyDeviceToHost, C.st));
            }
            NB_CK(cudaStreamSynchronize(C.st));
            tProject = std::chrono::duration<double>(nb::Clock::now() - t0).count() - tLayout;
        }
        catch (...)
        {
            status = nb::capi::StatusOf(std::current_exception());
            err = nb::capi::g_error;
            res.status = status;
            // a device error may leave the context unusable: the next request gets a fresh one
            ctx.reset();
        }
        const double ms =
            std::chrono::duration<double, std::milli>(nb::Clock::now() - q->submitted).count();
        {
            std::lock_guard<std::mutex> lock(mu);
            used[(size_t)dev] -= q->bytes;
            running--;
            layoutSeconds += tLayout;
            projectSeconds += tProject;
            nb::Record &rec = records[q->ticket];
            rec.state = 2;
            rec.status = status;
            rec.result = res;
            rec.result.latency_ms = ms;
            rec.error = err;
            if (status == NB_OK || status == NB_NOT_CONVERGED)
            {
                completed++;
                latencies.push_back(ms);
                doneOn[(size_t)dev]++;
            }
            else
                failed++;
        }
        cv.notify_all();
    }
}

using nb::capi::Fail;
using nb::capi::Guard;

extern "C" {

void nereus_b200_default_server_options(nb_server_options *o)
{
    if (!o) return;
    o->n_devices = 1;
    o->devices = nullptr;
    o->slots_per_device = 4;
    o->hbm_budget_gb = 150.0;
    nereus_b200_default_options(&o->solver);
}

int nereus_b200_server_create(nb_server **srv, const nb_server_options *opt)
{
    if (!srv) return Fail(NB_BAD_INPUT, "srv is null");
    *srv = nullptr;
    return Guard([&] {
        nb_server_options o;
        nereus_b200_default_server_options(&o);
        if (opt) o = *opt;
        if (o.n_devices < 1 || o.slots_per_device < 1 || !(o.hbm_budget_gb > 0.0))
            throw nb::InputError("n_devices, slots_per_device and hbm_budget_gb must be positive");
        int count = 0;
        NB_CK(cudaGetDeviceCount(&count));
        auto s = std::make_unique<nb_server>();
        s->opt = o;
        for (int d = 0; d < o.n_devices; d++)
        {
            const int dev = o.devices ? o.devices[d] : d;
            if (dev < 0 || dev >= count) throw nb::InputError("no such device");
            s->devices.push_back(dev);
        }
        s->opt.devices = nullptr;
        s->used.assign(s->devices.size(), 0.0);
        s->doneOn.assign(s->devices.size(), 0);
        s->budget = o.hbm_budget_gb * 1e9;
        for (size_t d = 0; d < s->devices.size(); d++)
            for (int k = 0; k < o.slots_per_device; k++) s->slots.emplace_back(&nb_server::Slot, s.get(), (int)d);
        *srv = s.release();
        return (int)NB_OK;
    });
}

void nereus_b200_server_destroy(nb_server *srv)
{
    if (!srv) return;
    {
        // the queued requests end unstarted; the running ones finish before their slots see `stop`
        std::lock_guard<std::mutex> lock(srv->mu);
        srv->queue.clear();
        srv->stop = true;
    }
    srv->cv.notify_all();
    for (auto &t : srv->slots)
        if (t.joinable()) t.join();
    delete srv;
}

int nereus_b200_submit(nb_server *srv, const nb_request *req, uint64_t *ticket)
{
    if (!srv || !req || !ticket) return Fail(NB_BAD_INPUT, "null argument");
    return Guard([&] {
        const nb_request &r = *req;
        if (r.dim != 2 && r.dim != 3) throw nb::InputError("dim must be 2 or 3");
        const int Nz = r.dim == 3 ? r.Nz : 1;
        if (r.Nx < 2 || r.Ny < 2 || Nz < 1 || (r.dim == 3 && Nz < 2)) throw nb::InputError("grid too small");
        if (!r.cell_types || !r.u || !r.v || !r.p || (r.dim == 3 && !r.w)) throw nb::InputError("null request field");
        for (int a = 0; a < r.dim; a++)
            if (!r.width[a] || !r.gap[a]) throw nb::InputError("null spacing table");
        if ((r.scheme == NB_SCHEME_INCREMENTAL || r.warm_start) && !r.p_prev)
            throw nb::InputError("the previous pressure is required");
        if (r.fields_on_device && srv->devices.size() != 1)
            throw nb::InputError("device-resident fields need a server of one device");
        auto q = std::make_unique<nb::Request>();
        q->r = r;
        q->r.Nz = Nz;
        const size_t cells = (size_t)r.Nx * r.Ny * Nz;
        q->types.assign(r.cell_types, r.cell_types + cells);
        const int N[3] = {r.Nx, r.Ny, Nz};
        for (int a = 0; a < 3; a++)
        {
            if (a == 2 && r.dim == 2)
            {
                // the 2D tables of z are never read; keep one-cell placeholders
                q->tables[2].assign(3, 1.0);
                q->tables[5].assign(2, 1.0);
                continue;
            }
            q->tables[a].assign(r.width[a], r.width[a] + N[a] + 2);
            q->tables[3 + a].assign(r.gap[a], r.gap[a] + N[a] + 1);
        }
        q->bytes = nb::RequestBytes(r.dim, r.Nx, r.Ny, Nz, srv->opt.solver.precision);
        if (q->bytes > srv->budget) throw nb::InputError("request larger than the device memory budget");
        {
            std::lock_guard<std::mutex> lock(srv->mu);
            if (srv->stop) throw nb::InputError("the server is stopping");
            q->ticket = srv->nextTicket++;
            q->submitted = nb::Clock::now();
            if (!srv->started)
            {
                srv->started = true;
                srv->first = q->submitted;
            }
            srv->records[q->ticket] = nb::Record{};
            srv->submitted++;
            *ticket = q->ticket;
            srv->queue.push_back(std::move(q));
        }
        srv->cv.notify_all();
        return (int)NB_OK;
    });
}

static int Report(nb_server *srv, const nb::Record &rec, nb_result *out)
{
    if (rec.state != 2) return NB_BUSY;
    if (out) *out = rec.result;
    if (rec.status != NB_OK && rec.status != NB_NOT_CONVERGED) Fail(rec.status, rec.error);
    return rec.status;
}

int nereus_b200_poll(nb_server *srv, uint64_t ticket, nb_result *out)
{
    if (!srv) return Fail(NB_BAD_INPUT, "srv is null");
    std::lock_guard<std::mutex> lock(srv->mu);
    auto it = srv->records.find(ticket);
    if (it == srv->records.end()) return Fail(NB_BAD_INPUT, "unknown ticket");
    return Report(srv, it->second, out);
}

int nereus_b200_wait(nb_server *srv, uint64_t ticket, double timeout_s, nb_result *out)
{
    if (!srv) return Fail(NB_BAD_INPUT, "srv is null");
    std::unique_lock<std::mutex> lock(srv->mu);
    auto it = srv->records.find(ticket);
    if (it == srv->records.end()) return Fail(NB_BAD_INPUT, "unknown ticket");
    auto done = [&] { return srv->records[ticket].state == 2; };
    if (timeout_s < 0.0) srv->cv.wait(lock, done);
    else srv->cv.wait_for(lock, std::chrono::duration<double>(timeout_s), done);
    return Report(srv, srv->records[ticket], out);
}

int nereus_b200_server_stats(nb_server *srv, nb_server_stats *st)
{
    if (!srv || !st) return Fail(NB_BAD_INPUT, "null argument");
    std::lock_guard<std::mutex> lock(srv->mu);
    *st = nb_server_stats{};
    st->submitted = srv->submitted;
    st->completed = srv->completed;
    st->failed = srv->failed;
    st->queued = (long long)srv->queue.size();
    st->running = srv->running;
    st->seconds = srv->started ? std::chrono::duration<double>(nb::Clock::now() - srv->first).count() : 0.0;
    st->solves_per_s = st->seconds > 0.0 ? (double)srv->completed / st->seconds : 0.0;
    if (!srv->latencies.empty())
    {
        std::vector<double> l = srv->latencies;
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) {
            const double k = (l.size() - 1) * q;
            const size_t lo = (size_t)k, hi = std::min(lo + 1, l.size() - 1);
            return l[lo] + (l[hi] - l[lo]) * (k - (double)lo);
        };
        st->p50_ms = pct(0.5);
        st->p99_ms = pct(0.99);
        double sum = 0.0;
        for (double x : l) sum += x;
        st->mean_ms = sum / (double)l.size();
    }
    double adm = 0.0;
    for (double u : srv->used) adm += u;
    st->admitted_gb = adm / 1e9;
    st->layout_s = srv->layoutSeconds;
    st->project_s = srv->projectSeconds;
    for (size_t d = 0; d < srv->doneOn.size() && d < 8; d++) st->device_completed[d] = srv->doneOn[d];
    return (int)NB_OK;
}

int nereus_b200_server_reset_stats(nb_server *srv)
{
    if (!srv) return Fail(NB_BAD_INPUT, "srv is null");
    std::lock_guard<std::mutex> lock(srv->mu);
    srv->submitted = (long long)srv->queue.size() + srv->running;
    srv->completed = srv->failed = 0;
    srv->latencies.clear();
    srv->layoutSeconds = srv->projectSeconds = 0.0;
    std::fill(srv->doneOn.begin(), srv->doneOn.end(), 0LL);
    srv->started = false;
    return (int)NB_OK;
}

double nereus_b200_request_bytes(int dim, int Nx, int Ny, int Nz, int precision)
{
    return nb::RequestBytes(dim, Nx, Ny, dim == 3 ? Nz : 1, precision);
}

int nereus_b200_plan(const double *costs, int n, int k, int *device_of)
{
    if (n < 0 || k < 1 || (n > 0 && (!costs || !device_of))) return Fail(NB_BAD_INPUT, "bad plan arguments");
    nb::Plan(costs, n, k, device_of);
    return (int)NB_OK;
}

} // extern "C"
