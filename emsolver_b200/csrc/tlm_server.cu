// tlm_server.cu -- continuous-batching request loop for antenna solves
// (C ABI tlm_server_*), built on the public handle and batch APIs.
//
// Callers submit complete solve requests (grid, materials, sources, probes,
// DFT frequencies). A worker thread owns one batch: between launch windows
// it admits queued requests -- the least work (cells x steps) first, or in
// arrival order -- while their HBM footprint fits the budget and the running
// cells stay within a target that keeps the GPU busy (state stays resident
// on the device until the request ends),
// attaches them to the running batch, advances every running request one
// window, and retires the requests that reached their total_steps: their
// port DFTs and records are copied out, the handle is freed and waiters are
// woken. Arrivals therefore overlap on the GPU with requests already
// running. Latency = completion time - submission time.
#include "tlm_b200.h"
#include "tlm_internal.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

struct PortSpec
{
    std::vector<uint64_t> cells;
    int pol;
    float amp;
};

struct Request
{
    uint64_t id = 0;
    // inputs (owned copies)
    tlm_grid grid{};
    std::vector<uint8_t> mat;
    std::vector<tlm_matprops> table;
    tlm_config cfg{};
    std::vector<float> sv;
    std::vector<PortSpec> ports;
    std::vector<int> probes;  // i j k per probe
    std::vector<double> freqs;
    size_t footprint = 0;
    long long nodes = 0;      // padded cells of the grid
    double work = 0.0;        // nodes x total_steps
    bool solo = false;        // stepped on its own stream by the single-grid kernels, not in the batch
    // progress
    int state = TLM_REQ_QUEUED;
    std::string error;
    Clock::time_point submitted, started, finished;
    tlm_handle h = nullptr;
    // results
    std::vector<std::vector<double>> dft;    // per port: Vre Vim Ire Iim interleaved by freq
    std::vector<std::vector<float>> vRec, iRec;
    std::vector<std::vector<float>> probeEz;
    int steps = 0;
};

} // namespace

struct tlm_server_s
{
    int device = 0;
    size_t budget = 0;
    size_t used = 0;
    int maxRunning = 1024;
    int window = 64;
    int order = TLM_SERVE_LEAST_WORK;   // admission order (tlm_server_set_policy)
    // Defaults measured on the served streams (Poisson 200/s; edges up to 128
    // and 256): with a cap of 8 Mi running cells and requests of 1 Mi cells
    // and up stepped on their own, p50 0.78-0.86 s / p99 3.8-3.9 s and 44
    // solves/s on the first against 2.4 s / 4.7 s and 38 with 32 Mi and 4 Mi;
    // p50 1.9 s / p99 14.4 s and 3.9 solves/s on the second against 4.6 s /
    // 16.8 s and 3.4.
    long long maxNodes = 8LL << 20;     // running cells cap (0: none)
    long long soloNodes = 1LL << 20;    // requests this large run alone beside the batch (0: never)
    tlm_batch batch = nullptr;
    std::mutex m;
    std::condition_variable cvWork, cvDone;
    std::deque<std::shared_ptr<Request>> queue;
    std::map<uint64_t, std::shared_ptr<Request>> all;
    std::vector<std::shared_ptr<Request>> running;
    std::vector<double> latencies;  // completed requests, seconds
    uint64_t nextId = 1;
    bool stop = false;
    std::thread worker;
    Clock::time_point t0;
    Clock::time_point lastDone;
    long long completed = 0, failed = 0, cancelledCount = 0;
    long long windows = 0;
    double busySeconds = 0.0;
    double gpuWindowSeconds = 0.0, setupSeconds = 0.0, retireSeconds = 0.0, cellWindows = 0.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string fatal;
};

namespace {

tlm_status serverFail(tlm_status s, const std::string &m)
{
    tlmi::setThreadError(m);
    return s;
}

// Device bytes a request holds while it runs (the figure tlm_setup admits
// against): two pulse buffers, stubs if any dielectric, the material map,
// records and monitors.
size_t footprintOf(const tlm_grid &g, const std::vector<uint8_t> &mat, const tlm_config &cfg,
                   size_t nports, size_t nprobes, size_t nfreq)
{
    const size_t px = (size_t)((g.nx + 7) / 8 * 8);
    const size_t P = px * g.ny * g.nz;
    const size_t sb = tlmi::storageBytes(cfg.storage);
    const size_t rb = cfg.storage == TLM_STORE_F64 ? 8 : 4;
    bool diel = false;
    for (uint8_t v : mat)
        if (v >= TLM_MAT_DIEL0)
        {
            diel = true;
            break;
        }
    const size_t steps = (size_t)std::max(cfg.total_steps, 1);
    return 2 * 12 * P * sb + (diel ? 3 * P * rb : 0) + P + steps * (nports * 2 + nprobes * 3 + 1) * 8 +
           nports * nfreq * 32 + steps * rb + (1u << 20);
}

// Cells of the near-field box a request will get (tlm_config.near_field):
// the bounding box of its PEC cells and port cells grown by the radius.
size_t nearCellsOf(const tlm_grid &g, const std::vector<uint8_t> &mat, const tlm_config &cfg,
                   const std::vector<PortSpec> &ports)
{
    if (cfg.near_field <= 0 || (cfg.storage != TLM_STORE_F16 && cfg.storage != TLM_STORE_BF16)) return 0;
    long long lo[3] = { g.nx, g.ny, g.nz }, hi[3] = { -1, -1, -1 };
    auto take = [&](long long c) {
        const long long v[3] = { c % g.nx, c / g.nx % g.ny, c / ((long long)g.nx * g.ny) };
        for (int a = 0; a < 3; ++a)
        {
            lo[a] = std::min(lo[a], v[a]);
            hi[a] = std::max(hi[a], v[a]);
        }
    };
    for (size_t c = 0; c < mat.size(); ++c)
        if (mat[c] == TLM_MAT_PEC) take((long long)c);
    for (const PortSpec &p : ports)
        for (uint64_t c : p.cells) take((long long)c);
    if (hi[0] < 0) return 0;
    const long long n[3] = { g.nx, g.ny, g.nz };
    size_t cells = 1;
    for (int a = 0; a < 3; ++a)
        cells *= (size_t)(std::min(hi[a] + cfg.near_field, n[a] - 1) - std::max(lo[a] - cfg.near_field, 0LL) + 1);
    return cells;
}

// Create and populate the handle of a request (worker thread; may run while
// a window of the batch is on the GPU: the handle has its own stream).
tlm_status startRequest(tlm_server_s *s, Request &r)
{
    tlm_status st = tlm_create(&r.h, s->device);
    if (st != TLM_OK)
    {
        r.error = tlm_last_error(nullptr);
        return st;
    }
    auto bad = [&](tlm_status e) {
        r.error = tlm_last_error(r.h);
        tlm_destroy(r.h);
        r.h = nullptr;
        return e;
    };
    if ((st = tlm_setup(r.h, &r.grid, r.mat.data(), r.mat.size(), r.table.data(), (int)r.table.size(),
                        &r.cfg)) != TLM_OK)
        return bad(st);
    if (!r.sv.empty() && (st = tlm_set_source_table(r.h, r.sv.data(), (int)r.sv.size())) != TLM_OK)
        return bad(st);
    for (const PortSpec &p : r.ports)
    {
        int idx = 0;
        if ((st = tlm_add_port(r.h, p.cells.data(), (int)p.cells.size(), p.pol, p.amp, &idx)) != TLM_OK)
            return bad(st);
    }
    for (size_t q = 0; q + 2 < r.probes.size(); q += 3)
    {
        int idx = 0;
        if ((st = tlm_add_probe_cell(r.h, r.probes[q], r.probes[q + 1], r.probes[q + 2], &idx)) != TLM_OK)
            return bad(st);
    }
    if (!r.freqs.empty() && (st = tlm_set_port_dft(r.h, r.freqs.data(), (int)r.freqs.size())) != TLM_OK)
        return bad(st);
    (void)s;
    return TLM_OK;
}

// Copy the results out of a finished request's handle and free it.
void finishRequest(tlm_server_s *s, Request &r)
{
    if (!r.solo) tlm_batch_detach(s->batch, r.h);
    r.steps = tlm_current_step(r.h);
    const int np = tlm_port_count(r.h);
    const int nf = (int)r.freqs.size();
    r.dft.assign(np, {});
    r.vRec.assign(np, {});
    r.iRec.assign(np, {});
    for (int p = 0; p < np; ++p)
    {
        std::vector<double> a(nf), b(nf), c(nf), d(nf);
        int n = 0;
        if (nf > 0) tlm_get_port_dft(r.h, p, a.data(), b.data(), c.data(), d.data(), nf, &n);
        r.dft[p].resize(4 * (size_t)nf);
        for (int f = 0; f < nf; ++f)
        {
            r.dft[p][4 * f + 0] = a[f];
            r.dft[p][4 * f + 1] = b[f];
            r.dft[p][4 * f + 2] = c[f];
            r.dft[p][4 * f + 3] = d[f];
        }
        r.vRec[p].resize(r.steps);
        r.iRec[p].resize(r.steps);
        tlm_get_port(r.h, p, r.vRec[p].data(), r.iRec[p].data(), r.steps, &n);
    }
    const int nq = tlm_probe_count(r.h);
    r.probeEz.assign(nq, {});
    for (int q = 0; q < nq; ++q)
    {
        r.probeEz[q].resize(r.steps);
        int n = 0;
        tlm_get_probe(r.h, q, nullptr, nullptr, r.probeEz[q].data(), r.steps, &n);
    }
    tlm_destroy(r.h);
    r.h = nullptr;
}

void retire(tlm_server_s *s, std::unique_lock<std::mutex> &lk)
{
    std::vector<std::shared_ptr<Request>> keep;
    for (auto &r : s->running)
    {
        const bool done = tlm_current_step(r->h) >= r->cfg.total_steps;
        if (!done && r->state != TLM_REQ_CANCELLED)
        {
            keep.push_back(r);
            continue;
        }
        lk.unlock();
        if (done)
            finishRequest(s, *r);
        else
        {
            if (!r->solo) tlm_batch_detach(s->batch, r->h);
            tlm_destroy(r->h);
            r->h = nullptr;
        }
        lk.lock();
        r->finished = Clock::now();
        s->used -= r->footprint;
        if (done && r->state != TLM_REQ_CANCELLED)
        {
            r->state = TLM_REQ_DONE;
            ++s->completed;
            s->latencies.push_back(std::chrono::duration<double>(r->finished - r->submitted).count());
            s->lastDone = r->finished;
        }
    }
    s->running.swap(keep);
}

// The worker: per iteration, pick the queued requests that fit the budget,
// launch one window for the running ones, set the picked ones up while the
// GPU works, wait for the window, retire finished requests and attach the
// new ones, which take part from the next window on.
void workerMain(tlm_server_s *s)
{
    std::unique_lock<std::mutex> lk(s->m);
    while (true)
    {
        std::vector<std::shared_ptr<Request>> picked;
        size_t planned = s->used;
        long long plannedNodes = 0;
        for (const auto &r : s->running) plannedNodes += r->nodes;
        while (!s->stop && !s->queue.empty() &&
               (int)(s->running.size() + picked.size()) < s->maxRunning)
        {
            // the next candidate: the least work, or the oldest request
            auto it = s->queue.begin();
            if (s->order == TLM_SERVE_LEAST_WORK)
                it = std::min_element(s->queue.begin(), s->queue.end(),
                                      [](const std::shared_ptr<Request> &a, const std::shared_ptr<Request> &b) {
                                          return a->work < b->work || (a->work == b->work && a->id < b->id);
                                      });
            std::shared_ptr<Request> r = *it;
            if (r->state == TLM_REQ_CANCELLED)
            {
                s->queue.erase(it);
                continue;
            }
            const bool first = s->running.empty() && picked.empty();
            if (planned + r->footprint > s->budget && !first) break;
            if (s->maxNodes > 0 && plannedNodes + r->nodes > s->maxNodes && !first) break;
            s->queue.erase(it);
            plannedNodes += r->nodes;
            r->state = TLM_REQ_RUNNING;
            r->started = Clock::now();
            planned += r->footprint;
            s->used += r->footprint;
            picked.push_back(r);
        }
        if (s->stop)
        {
            for (auto &r : picked)
            {
                r->state = TLM_REQ_CANCELLED;
                s->used -= r->footprint;
            }
            break;
        }
        if (s->running.empty() && picked.empty())
        {
            s->cvWork.wait(lk, [&] { return s->stop || !s->queue.empty(); });
            continue;
        }
        std::vector<tlm_handle> solos;
        bool haveBatch = false;
        long long runningCells = 0;
        for (const auto &r : s->running)
        {
            runningCells += r->nodes;
            if (r->solo)
                solos.push_back(r->h);
            else
                haveBatch = true;
        }
        const bool haveRunning = haveBatch;
        const int soloWindow = s->window;
        lk.unlock();
        const Clock::time_point w0 = Clock::now();
        int launched = 0;
        tlm_status st = TLM_OK;
        void *bs = nullptr;
        tlm_batch_get_stream(s->batch, &bs);
        if (haveRunning && s->ev0) cudaEventRecord(s->ev0, static_cast<cudaStream_t>(bs));
        if (haveRunning) st = tlm_batch_launch_window(s->batch, &launched);
        if (haveRunning && s->ev1) cudaEventRecord(s->ev1, static_cast<cudaStream_t>(bs));
        // large requests: one window each on their own stream, beside the batch
        for (tlm_handle h : solos)
        {
            const int left = tlm_total_steps(h) - tlm_current_step(h);
            if (st == TLM_OK && left > 0) st = tlm_step_async(h, std::min(left, soloWindow));
            if (left > 0) launched = std::max(launched, 1);
        }
        const Clock::time_point p0 = Clock::now();
        std::vector<tlm_status> prep(picked.size(), TLM_OK);
        for (size_t k = 0; k < picked.size(); ++k) prep[k] = startRequest(s, *picked[k]);
        const double setupDt = std::chrono::duration<double>(Clock::now() - p0).count();
        if (st == TLM_OK && haveRunning) st = tlm_batch_sync(s->batch);
        for (tlm_handle h : solos)
            if (st == TLM_OK) st = tlm_sync(h);
        const double dt = std::chrono::duration<double>(Clock::now() - w0).count();
        float gpuMs = 0.0f;
        if (launched && s->ev0 && cudaEventElapsedTime(&gpuMs, s->ev0, s->ev1) != cudaSuccess)
        {
            cudaGetLastError();
            gpuMs = 0.0f;
        }
        lk.lock();
        s->setupSeconds += setupDt;
        if (launched)
        {
            s->busySeconds += dt;
            s->gpuWindowSeconds += gpuMs * 1e-3;
            s->cellWindows += (double)runningCells;
            ++s->windows;
        }
        if (st != TLM_OK)
        {
            s->fatal = tlm_last_error(nullptr);
            for (auto &r : s->running)
            {
                r->state = TLM_REQ_FAILED;
                r->error = s->fatal;
                r->finished = Clock::now();
                if (!r->solo) tlm_batch_detach(s->batch, r->h);
                tlm_destroy(r->h);
                r->h = nullptr;
                ++s->failed;
                s->used -= r->footprint;
            }
            s->running.clear();
        }
        else
        {
            const Clock::time_point r0 = Clock::now();
            retire(s, lk);
            s->retireSeconds += std::chrono::duration<double>(Clock::now() - r0).count();
        }
        // attach the requests set up during this window
        for (size_t k = 0; k < picked.size(); ++k)
        {
            Request &r = *picked[k];
            tlm_status ps = prep[k];
            if (ps == TLM_OK && r.state == TLM_REQ_CANCELLED)
            {
                tlm_destroy(r.h);
                r.h = nullptr;
                s->used -= r.footprint;
                r.finished = Clock::now();
                continue;
            }
            r.solo = s->soloNodes > 0 && r.nodes >= s->soloNodes;
            if (ps == TLM_OK && !r.solo && (ps = tlm_batch_attach(s->batch, r.h)) != TLM_OK)
            {
                r.error = tlm_last_error(nullptr);
                tlm_destroy(r.h);
                r.h = nullptr;
            }
            if (ps == TLM_ENOMEM && !s->running.empty())
            {
                // the device is fuller than the budget says: retry this
                // request once a running one has freed its memory
                r.state = TLM_REQ_QUEUED;
                r.error.clear();
                s->used -= r.footprint;
                s->queue.push_front(picked[k]);
                continue;
            }
            if (ps != TLM_OK)
            {
                r.state = TLM_REQ_FAILED;
                r.finished = Clock::now();
                s->used -= r.footprint;
                ++s->failed;
                continue;
            }
            s->running.push_back(picked[k]);
        }
        s->cvDone.notify_all();
    }
    // shutdown: cancel what is left
    for (auto &r : s->running)
    {
        if (!r->solo) tlm_batch_detach(s->batch, r->h);
        tlm_destroy(r->h);
        r->h = nullptr;
        r->state = TLM_REQ_CANCELLED;
    }
    s->running.clear();
    for (auto &r : s->queue) r->state = TLM_REQ_CANCELLED;
    s->queue.clear();
    s->cvDone.notify_all();
}

double percentile(std::vector<double> v, double p)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = p * (double)(v.size() - 1);
    const size_t lo = (size_t)pos, hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (pos - (double)lo) * (v[hi] - v[lo]);
}

} // namespace

extern "C" {

tlm_status tlm_server_create(tlm_server *out, int device, size_t hbm_budget_bytes, int steps_per_launch)
{
    if (!out) return serverFail(TLM_EINVAL, "null output");
    *out = nullptr;
    auto *s = new tlm_server_s();
    s->device = device;
    s->window = steps_per_launch > 0 ? steps_per_launch : 64;
    tlm_status st = tlm_batch_create(&s->batch, device);
    if (st != TLM_OK)
    {
        delete s;
        return st;
    }
    tlm_batch_tuning t{ 0, s->window, 0, 1, 0, 0.0 };
    tlm_batch_set_tuning(s->batch, &t);
    if (hbm_budget_bytes == 0)
    {
        size_t freeB = 0, totalB = 0;
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        cudaMemGetInfo(&freeB, &totalB);
        cudaSetDevice(prev);
        hbm_budget_bytes = freeB / 10 * 8;
    }
    s->budget = hbm_budget_bytes;
    {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        if (cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess)
        {
            cudaGetLastError();
            s->ev0 = s->ev1 = nullptr;
        }
        cudaSetDevice(prev);
    }
    s->t0 = Clock::now();
    s->lastDone = s->t0;
    s->worker = std::thread(workerMain, s);
    *out = s;
    return TLM_OK;
}

tlm_status tlm_server_set_policy(tlm_server s, int order, long long max_running_cells, long long solo_cells)
{
    if (!s) return serverFail(TLM_EINVAL, "null server");
    if (order != TLM_SERVE_ARRIVAL && order != TLM_SERVE_LEAST_WORK)
        return serverFail(TLM_EINVAL, "order must be TLM_SERVE_ARRIVAL or TLM_SERVE_LEAST_WORK");
    if (max_running_cells < 0 || solo_cells < 0)
        return serverFail(TLM_EINVAL, "max_running_cells and solo_cells must be >= 0");
    std::lock_guard<std::mutex> lk(s->m);
    s->order = order;
    s->maxNodes = max_running_cells;
    s->soloNodes = solo_cells;
    return TLM_OK;
}

tlm_status tlm_server_destroy(tlm_server s)
{
    if (!s) return TLM_OK;
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->stop = true;
    }
    s->cvWork.notify_all();
    if (s->worker.joinable()) s->worker.join();
    tlm_batch_destroy(s->batch);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    delete s;
    return TLM_OK;
}

tlm_status tlm_server_submit(tlm_server s, const tlm_request *q, uint64_t *id)
{
    if (!s || !q || !id) return serverFail(TLM_EINVAL, "null server, request or id");
    if (!q->mat || q->n_cells != (size_t)q->grid.nx * q->grid.ny * q->grid.nz)
        return serverFail(TLM_EINVAL, "material map does not match the grid");
    if (q->n_ports < 0 || q->n_probes < 0 || q->n_freq < 0 || q->n_table < 0 || q->n_source < 0)
        return serverFail(TLM_EINVAL, "negative count");
    if (q->cfg.surface_monitors || q->cfg.record_every)
        return serverFail(TLM_EINVAL, "served requests record ports and probes only "
                                      "(surface_monitors = 0, record_every = 0)");
    auto r = std::make_shared<Request>();
    r->grid = q->grid;
    r->mat.assign(q->mat, q->mat + q->n_cells);
    if (q->n_table) r->table.assign(q->table, q->table + q->n_table);
    r->cfg = q->cfg;
    if (q->n_source) r->sv.assign(q->source_table, q->source_table + q->n_source);
    size_t off = 0;
    for (int p = 0; p < q->n_ports; ++p)
    {
        PortSpec ps;
        ps.cells.assign(q->port_cells + off, q->port_cells + off + q->port_ncells[p]);
        off += q->port_ncells[p];
        ps.pol = q->port_pol[p];
        ps.amp = q->port_amp[p];
        r->ports.push_back(std::move(ps));
    }
    if (q->n_probes) r->probes.assign(q->probe_ijk, q->probe_ijk + 3 * (size_t)q->n_probes);
    if (q->n_freq) r->freqs.assign(q->freqs, q->freqs + q->n_freq);
    r->footprint = footprintOf(r->grid, r->mat, r->cfg, r->ports.size(), (size_t)q->n_probes,
                               r->freqs.size()) +
                   2 * 12 * sizeof(float) * nearCellsOf(r->grid, r->mat, r->cfg, r->ports);
    r->nodes = (long long)((r->grid.nx + 7) / 8 * 8) * r->grid.ny * r->grid.nz;
    r->work = (double)r->nodes * (double)std::max(r->cfg.total_steps, 1);
    std::lock_guard<std::mutex> lk(s->m);
    if (s->stop) return serverFail(TLM_ESTATE, "the server is shutting down");
    if (r->footprint > s->budget)
        return serverFail(TLM_ENOMEM, "request needs " + std::to_string(r->footprint >> 20) +
                                          " MiB, the server budget is " + std::to_string(s->budget >> 20) +
                                          " MiB");
    r->id = s->nextId++;
    r->submitted = Clock::now();
    s->queue.push_back(r);
    s->all[r->id] = r;
    *id = r->id;
    s->cvWork.notify_one();
    return TLM_OK;
}

tlm_status tlm_server_poll(tlm_server s, uint64_t id, int *state)
{
    if (!s || !state) return serverFail(TLM_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(s->m);
    auto it = s->all.find(id);
    if (it == s->all.end()) return serverFail(TLM_EINVAL, "unknown request id");
    *state = it->second->state;
    return TLM_OK;
}

tlm_status tlm_server_wait(tlm_server s, uint64_t id, double timeout_s, int *state)
{
    if (!s) return serverFail(TLM_EINVAL, "null server");
    std::unique_lock<std::mutex> lk(s->m);
    auto it = s->all.find(id);
    if (it == s->all.end()) return serverFail(TLM_EINVAL, "unknown request id");
    auto r = it->second;
    auto ended = [&] {
        return r->state == TLM_REQ_DONE || r->state == TLM_REQ_FAILED || r->state == TLM_REQ_CANCELLED;
    };
    if (timeout_s < 0)
        s->cvDone.wait(lk, ended);
    else if (!s->cvDone.wait_for(lk, std::chrono::duration<double>(timeout_s), ended))
    {
        if (state) *state = r->state;
        return serverFail(TLM_ETIMEOUT, "request still running");
    }
    if (state) *state = r->state;
    return TLM_OK;
}

tlm_status tlm_server_cancel(tlm_server s, uint64_t id)
{
    if (!s) return serverFail(TLM_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(s->m);
    auto it = s->all.find(id);
    if (it == s->all.end()) return serverFail(TLM_EINVAL, "unknown request id");
    Request &r = *it->second;
    if (r.state == TLM_REQ_QUEUED || r.state == TLM_REQ_RUNNING)
    {
        const bool queued = r.state == TLM_REQ_QUEUED;
        r.state = TLM_REQ_CANCELLED;
        ++s->cancelledCount;
        if (queued) r.finished = Clock::now();
    }
    s->cvDone.notify_all();
    return TLM_OK;
}

tlm_status tlm_server_result(tlm_server s, uint64_t id, int port, double *v_re, double *v_im,
                             double *i_re, double *i_im, int cap, int *n_freq, double *latency_s)
{
    if (!s) return serverFail(TLM_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(s->m);
    auto it = s->all.find(id);
    if (it == s->all.end()) return serverFail(TLM_EINVAL, "unknown request id");
    Request &r = *it->second;
    if (r.state == TLM_REQ_FAILED) return serverFail(TLM_ECUDA, "request failed: " + r.error);
    if (r.state != TLM_REQ_DONE) return serverFail(TLM_ESTATE, "request not finished");
    if (port < 0 || port >= (int)r.dft.size()) return serverFail(TLM_EINVAL, "port index out of range");
    const int nf = (int)r.freqs.size();
    if (n_freq) *n_freq = nf;
    for (int f = 0; f < nf && f < cap; ++f)
    {
        if (v_re) v_re[f] = r.dft[port][4 * f + 0];
        if (v_im) v_im[f] = r.dft[port][4 * f + 1];
        if (i_re) i_re[f] = r.dft[port][4 * f + 2];
        if (i_im) i_im[f] = r.dft[port][4 * f + 3];
    }
    if (latency_s) *latency_s = std::chrono::duration<double>(r.finished - r.submitted).count();
    return TLM_OK;
}

tlm_status tlm_server_port_records(tlm_server s, uint64_t id, int port, float *v, float *i, int cap,
                                   int *n_out)
{
    if (!s) return serverFail(TLM_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(s->m);
    auto it = s->all.find(id);
    if (it == s->all.end()) return serverFail(TLM_EINVAL, "unknown request id");
    Request &r = *it->second;
    if (r.state != TLM_REQ_DONE) return serverFail(TLM_ESTATE, "request not finished");
    if (port < 0 || port >= (int)r.vRec.size()) return serverFail(TLM_EINVAL, "port index out of range");
    if (n_out) *n_out = r.steps;
    for (int t = 0; t < r.steps && t < cap; ++t)
    {
        if (v) v[t] = r.vRec[port][t];
        if (i) i[t] = r.iRec[port][t];
    }
    return TLM_OK;
}

tlm_status tlm_server_release(tlm_server s, uint64_t id)
{
    if (!s) return serverFail(TLM_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(s->m);
    auto it = s->all.find(id);
    if (it == s->all.end()) return serverFail(TLM_EINVAL, "unknown request id");
    const int st = it->second->state;
    if (st == TLM_REQ_QUEUED || st == TLM_REQ_RUNNING) return serverFail(TLM_ESTATE, "request still active");
    s->all.erase(it);
    return TLM_OK;
}

tlm_status tlm_server_stats(tlm_server s, tlm_server_stats_t *out)
{
    if (!s || !out) return serverFail(TLM_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(s->m);
    std::memset(out, 0, sizeof(*out));
    out->completed = s->completed;
    out->failed = s->failed;
    out->cancelled = s->cancelledCount;
    out->queued = (long long)s->queue.size();
    out->running = (long long)s->running.size();
    out->latency_p50_s = percentile(s->latencies, 0.50);
    out->latency_p99_s = percentile(s->latencies, 0.99);
    out->latency_mean_s = 0.0;
    for (double l : s->latencies) out->latency_mean_s += l;
    if (!s->latencies.empty()) out->latency_mean_s /= (double)s->latencies.size();
    const double span = std::chrono::duration<double>(s->lastDone - s->t0).count();
    out->solves_per_s = span > 0 ? (double)s->completed / span : 0.0;
    out->hbm_used_bytes = s->used;
    out->hbm_budget_bytes = s->budget;
    out->windows = s->windows;
    out->busy_s = s->busySeconds;
    out->gpu_window_s = s->gpuWindowSeconds;
    out->setup_s = s->setupSeconds;
    out->retire_s = s->retireSeconds;
    out->mean_running_cells = s->windows ? s->cellWindows / (double)s->windows : 0.0;
    return TLM_OK;
}

tlm_status tlm_request_footprint(const tlm_request *q, size_t *bytes)
{
    if (!q || !bytes || !q->mat) return serverFail(TLM_EINVAL, "null argument");
    std::vector<uint8_t> m(q->mat, q->mat + q->n_cells);
    std::vector<PortSpec> ports;
    size_t off = 0;
    for (int p = 0; p < q->n_ports; ++p)
    {
        PortSpec ps;
        ps.cells.assign(q->port_cells + off, q->port_cells + off + q->port_ncells[p]);
        off += q->port_ncells[p];
        ports.push_back(std::move(ps));
    }
    *bytes = footprintOf(q->grid, m, q->cfg, (size_t)q->n_ports, (size_t)q->n_probes, (size_t)q->n_freq) +
             2 * 12 * sizeof(float) * nearCellsOf(q->grid, m, q->cfg, ports);
    return TLM_OK;
}

} // extern "C"
