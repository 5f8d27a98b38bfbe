// serve.cu — continuous batching of simulation requests over one or more
// contexts (one per GPU).
//
// Requests queue on submit (their host data is copied).  Each tick:
//   1. retire requests that finished or were cancelled;
//   2. admit queued requests, first come first served: the request at the
//      head of the queue goes to the context with the most unused budget
//      among those where it fits (slot limit, device-memory budget, the
//      running set's time step); admission stops at the first request
//      that fits nowhere;
//   3. on each context whose running set changed, build a new batch over
//      it: requests that keep running move their fields and cells
//      device-to-device from the old batch, new ones upload their inputs;
//   4. advance every running request by min(steps_per_tick, fewest steps
//      left) main-loop sub-steps -- each sub-step is one graph launch over
//      a context's requests, with a per-request mask so that every request
//      keeps its own mechanics cadence (src/main.mm:375-391 accumulator);
//      all contexts' launches are issued before any is waited for, so the
//      GPUs work at the same time;
//   5. requests that reached their step count copy their results to the
//      host and leave at the next tick.
// A request's arithmetic never depends on what else runs or where (every
// kernel treats instances independently and in a fixed order), so its
// result is the same alone and in the mix, on any context.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <new>
#include <vector>

#include "batch.h"

using namespace pcg;

namespace {

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    uint64_t id = 0;
    pcg_instance_desc desc{};
    std::vector<pcg_substrate_params> subs;
    std::vector<float> dens, init_vals, soa;
    std::vector<double> rates[4];
    std::vector<uint8_t> active;
    uint32_t n_steps = 0, done = 0;
    double accum = 0.0;
    int state = PCG_REQ_QUEUED;
    double t_submit = 0, t_admit = 0, t_done = 0;
    uint64_t bytes = 0;
    int lane = -1;   // context the request runs on
    int slot = -1;   // index in that context's current batch
    std::vector<float> out_dens, out_soa;
};

// One context of the server: its running set and their batch.
struct Lane {
    pcg_ctx* ctx = nullptr;
    std::vector<Request*> running;
    std::unique_ptr<Batch> batch;
    uint64_t bytes_in_use = 0;
    HostBuf masks;
    bool changed = false;
    uint32_t k = 0;   // sub-steps issued this tick
};

// Makes a device current for the life of the guard.
class DeviceScope {
public:
    explicit DeviceScope(int device)
    {
        if (cudaGetDevice(&prev_) == cudaSuccess && prev_ != device && cudaSetDevice(device) == cudaSuccess)
            switched_ = true;
    }
    ~DeviceScope()
    {
        if (switched_) cudaSetDevice(prev_);
    }
private:
    int prev_ = -1;
    bool switched_ = false;
};

}  // namespace

struct pcg_server {
    pcg_ctx* ctx = nullptr;   // the first context (error messages of server-wide calls)
    pcg_serve_options opt{};
    uint64_t next_id = 1;
    std::map<uint64_t, std::unique_ptr<Request>> reqs;
    std::deque<Request*> queue;
    std::vector<std::unique_ptr<Lane>> lanes;
    uint64_t voxel_steps = 0, cell_steps = 0;
};

namespace {

int rebuild(Lane& L)
{
    if (L.running.empty()) {
        L.batch.reset();
        return PCG_OK;
    }
    std::vector<pcg_instance_desc> descs;
    std::vector<DevSource> src;
    for (Request* r : L.running) {
        descs.push_back(r->desc);
        DevSource ds;
        if (r->slot >= 0 && L.batch) {
            ds.batch = L.batch.get();
            ds.index = static_cast<uint32_t>(r->slot);
        }
        src.push_back(ds);
    }
    pcg_batch_options o{};
    o.use_graphs = 1;
    o.autotune = 0;   // cached or default shapes: rebuilds must stay cheap
    std::unique_ptr<Batch> nb(new (std::nothrow) Batch());
    if (!nb) return PCG_ERR_OOM;
    PCG_TRY(nb->create(L.ctx, descs.data(), static_cast<uint32_t>(descs.size()), &o, &src, true));
    PCG_CU(L.ctx, cudaStreamSynchronize(L.ctx->stream));
    L.batch = std::move(nb);   // frees the old batch
    for (size_t i = 0; i < L.running.size(); ++i) L.running[i]->slot = static_cast<int>(i);
    return PCG_OK;
}

int finish(Lane& L, Request* r)
{
    Batch& b = *L.batch;
    const uint32_t i = static_cast<uint32_t>(r->slot);
    const DiffInstance& di = b.d.inst[i];
    r->out_dens.resize(di.nvox() * di.g.n_substrates);
    PCG_TRY(b.d.download(i, r->out_dens.data()));
    const CellInst& ci = b.c_.h_inst[i];
    r->out_soa.assign(static_cast<size_t>(NUM_FIELDS) * std::max<uint32_t>(ci.n_cells, 1), 0.f);
    if (ci.n_cells) {
        PCG_TRY(b.c_.download_soa(ci.cell_off, ci.n_cells, r->out_soa.data(), ci.n_cells, 0, NUM_FIELDS));
        PCG_CU(L.ctx, cudaStreamSynchronize(L.ctx->stream));
    }
    r->state = PCG_REQ_DONE;
    r->t_done = now_s();
    L.bytes_in_use -= r->bytes;
    return PCG_OK;
}

// Unused budget of a lane for a request, or -1 when it cannot take it now.
int64_t room_for(const pcg_server* s, const Lane& L, const Request* r)
{
    if (s->opt.max_active && L.running.size() >= s->opt.max_active) return -1;
    if (L.bytes_in_use + r->bytes > s->opt.budget_bytes) return -1;
    if (!L.running.empty() && L.running[0]->desc.grid.dt != r->desc.grid.dt) return -1;   // one time step per set
    return static_cast<int64_t>(s->opt.budget_bytes - L.bytes_in_use);
}

}  // namespace

extern "C" {

pcg_status pcg_serve_create_multi(pcg_ctx* const* ctxs, uint32_t n_ctx, const pcg_serve_options* opt,
                                  pcg_server** out)
{
    if (!ctxs || n_ctx == 0 || !out) return PCG_ERR_INVALID;
    for (uint32_t i = 0; i < n_ctx; ++i)
        if (!ctxs[i]) return PCG_ERR_INVALID;
    *out = nullptr;
    pcg_server* s = new (std::nothrow) pcg_server();
    if (!s) return PCG_ERR_OOM;
    s->ctx = ctxs[0];
    if (opt) s->opt = *opt;
    if (s->opt.budget_bytes == 0) s->opt.budget_bytes = 150ull * 1000 * 1000 * 1000;
    if (s->opt.steps_per_tick == 0) s->opt.steps_per_tick = 100;
    for (uint32_t i = 0; i < n_ctx; ++i) {
        std::unique_ptr<Lane> L(new (std::nothrow) Lane());
        if (!L) {
            delete s;
            return PCG_ERR_OOM;
        }
        L->ctx = ctxs[i];
        s->lanes.push_back(std::move(L));
    }
    for (auto& L : s->lanes) ctx_retain(L->ctx);
    *out = s;
    return PCG_OK;
}

pcg_status pcg_serve_create(pcg_ctx* ctx, const pcg_serve_options* opt, pcg_server** out)
{
    if (!ctx) return PCG_ERR_INVALID;
    return pcg_serve_create_multi(&ctx, 1, opt, out);
}

pcg_status pcg_serve_destroy(pcg_server* s)
{
    if (!s) return PCG_OK;
    std::vector<pcg_ctx*> ctxs;
    for (auto& L : s->lanes) {
        DeviceScope dev(L->ctx->device);
        cudaStreamSynchronize(L->ctx->stream);
        L->batch.reset();
        L->masks.release();
        ctxs.push_back(L->ctx);
    }
    delete s;
    for (pcg_ctx* c : ctxs) ctx_release(c);
    return PCG_OK;
}

pcg_status pcg_serve_submit(pcg_server* s, const pcg_instance_desc* in, uint32_t n_steps, uint64_t* id)
{
    if (!s || !in || !id) return PCG_ERR_INVALID;
    const pcg_instance_desc& d = *in;
    if (d.grid.nx == 0 || d.grid.ny == 0 || d.grid.nz == 0) return fail(s->ctx, PCG_ERR_INVALID, "empty grid");
    if (d.grid.n_substrates > 0 && !d.substrates) return fail(s->ctx, PCG_ERR_INVALID, "substrates is NULL");
    if (d.n_cells > 0 && (!d.cells_soa || d.cells_soa_max < d.n_cells))
        return fail(s->ctx, PCG_ERR_INVALID, "cells_soa missing or too small");
    std::unique_ptr<Request> r(new (std::nothrow) Request());
    if (!r) return PCG_ERR_OOM;
    r->bytes = instance_bytes(d);
    if (r->bytes > s->opt.budget_bytes) return fail(s->ctx, PCG_ERR_BUDGET, "request larger than the budget");
    r->id = s->next_id++;
    r->n_steps = n_steps;
    r->t_submit = now_s();
    r->desc = d;
    const uint32_t S = d.grid.n_substrates;
    const size_t nv = static_cast<size_t>(d.grid.nx) * d.grid.ny * d.grid.nz;
    r->subs.assign(d.substrates, d.substrates + S);
    r->desc.substrates = r->subs.data();
    if (d.initial_density) {
        r->dens.assign(d.initial_density, d.initial_density + nv * S);
        r->desc.initial_density = r->dens.data();
    }
    if (d.initial_values) {
        r->init_vals.assign(d.initial_values, d.initial_values + S);
        r->desc.initial_values = r->init_vals.data();
    }
    if (d.n_cells) {
        r->soa.resize(static_cast<size_t>(NUM_FIELDS) * d.n_cells);
        for (int f = 0; f < NUM_FIELDS; ++f)
            std::memcpy(r->soa.data() + static_cast<size_t>(f) * d.n_cells,
                        d.cells_soa + static_cast<size_t>(f) * d.cells_soa_max, d.n_cells * sizeof(float));
        r->desc.cells_soa = r->soa.data();
        r->desc.cells_soa_max = d.n_cells;
        const double* src[4] = {d.secretion, d.uptake, d.saturation, d.net_export};
        const double** dst[4] = {&r->desc.secretion, &r->desc.uptake, &r->desc.saturation, &r->desc.net_export};
        for (int q = 0; q < 4; ++q) {
            if (src[q]) {
                r->rates[q].assign(src[q], src[q] + static_cast<size_t>(d.n_cells) * S);
                *dst[q] = r->rates[q].data();
            } else {
                *dst[q] = nullptr;
            }
        }
        if (d.active) {
            r->active.assign(d.active, d.active + d.n_cells);
            r->desc.active = r->active.data();
        }
    }
    *id = r->id;
    s->queue.push_back(r.get());
    s->reqs[r->id] = std::move(r);
    return PCG_OK;
}

pcg_status pcg_serve_tick(pcg_server* s, uint32_t* n_running, uint32_t* n_queued, uint32_t* n_finished)
{
    if (!s) return PCG_ERR_INVALID;
    uint32_t finished = 0, running = 0;
    // 1. retire requests that finished in the previous tick or were cancelled
    for (auto& Lp : s->lanes) {
        Lane& L = *Lp;
        L.changed = false;
        std::vector<Request*> keep;
        for (Request* r : L.running) {
            if (r->state == PCG_REQ_DONE || r->state == PCG_REQ_CANCELLED) {
                L.changed = true;
                if (r->state == PCG_REQ_CANCELLED) L.bytes_in_use -= r->bytes;   // a finished one gave it back
                r->slot = -1;
            } else {
                keep.push_back(r);
            }
        }
        L.running.swap(keep);
    }
    // 2. admit, first come first served, each to the context with the most room
    while (!s->queue.empty()) {
        Request* r = s->queue.front();
        Lane* best = nullptr;
        int64_t best_room = -1;
        for (auto& Lp : s->lanes) {
            const int64_t room = room_for(s, *Lp, r);
            if (room > best_room) {
                best_room = room;
                best = Lp.get();
            }
        }
        if (!best) break;
        s->queue.pop_front();
        r->state = PCG_REQ_RUNNING;
        r->t_admit = now_s();
        for (size_t i = 0; i < s->lanes.size(); ++i)
            if (s->lanes[i].get() == best) r->lane = static_cast<int>(i);
        r->slot = -1;
        best->bytes_in_use += r->bytes;
        best->running.push_back(r);
        best->changed = true;
    }
    // 3. new batches where the running set changed
    for (auto& Lp : s->lanes) {
        Lane& L = *Lp;
        if (!L.changed) continue;
        DeviceScope dev(L.ctx->device);
        PCG_TRY(rebuild(L));
    }
    // 4. issue every context's sub-steps, then wait for all of them
    for (auto& Lp : s->lanes) {
        Lane& L = *Lp;
        L.k = 0;
        if (L.running.empty()) continue;
        DeviceScope dev(L.ctx->device);
        Batch& b = *L.batch;
        uint32_t k = 0;
        for (Request* r : L.running) k = std::max(k, std::min(s->opt.steps_per_tick, r->n_steps - r->done));
        const size_t n = L.running.size();
        if (L.masks.bytes < static_cast<size_t>(k) * n) {
            PCG_CU(L.ctx, cudaStreamSynchronize(L.ctx->stream));   // the old masks may still be read
            PCG_CU(L.ctx, L.masks.alloc(static_cast<size_t>(k) * n));
        }
        uint8_t* m = L.masks.as<uint8_t>();
        for (uint32_t st = 0; st < k; ++st) {
            bool any = false;
            for (size_t i = 0; i < n; ++i) {
                Request* r = L.running[i];
                if (r->done + st >= r->n_steps) {
                    m[st * n + i] = 0;
                    continue;
                }
                const double dtd = r->desc.grid.dt;
                const double dtm = r->desc.dt_mechanics > 0.f ? r->desc.dt_mechanics : r->desc.mech.dt;
                r->accum += dtd;
                const bool mech = r->accum >= dtm - 0.5 * dtd;
                if (mech) {
                    r->accum = 0.0;
                    any = true;
                    s->cell_steps += r->desc.n_cells;
                }
                m[st * n + i] = static_cast<uint8_t>(STEP_DIFFUSE | (mech ? STEP_MECH : 0));
            }
            PCG_TRY(b.step_masked(m + st * n, any));
        }
        L.k = k;
    }
    // 5. results of the requests that reached their step count
    for (auto& Lp : s->lanes) {
        Lane& L = *Lp;
        if (L.running.empty()) continue;
        DeviceScope dev(L.ctx->device);
        PCG_CU(L.ctx, cudaStreamSynchronize(L.ctx->stream));
        for (Request* r : L.running) {
            const uint32_t taken = std::min(L.k, r->n_steps - r->done);
            r->done += taken;
            s->voxel_steps += static_cast<uint64_t>(r->desc.grid.nx) * r->desc.grid.ny * r->desc.grid.nz * taken;
            if (r->done >= r->n_steps) {
                PCG_TRY(finish(L, r));
                ++finished;
            }
        }
        running += static_cast<uint32_t>(L.running.size());
    }
    if (n_running) *n_running = running - finished;
    if (n_queued) *n_queued = static_cast<uint32_t>(s->queue.size());
    if (n_finished) *n_finished = finished;
    return PCG_OK;
}

pcg_status pcg_serve_cancel(pcg_server* s, uint64_t id)
{
    if (!s) return PCG_ERR_INVALID;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return PCG_ERR_NOT_FOUND;
    Request* r = it->second.get();
    switch (r->state) {
    case PCG_REQ_QUEUED:
        s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
        r->state = PCG_REQ_CANCELLED;
        return PCG_OK;
    case PCG_REQ_RUNNING:
        r->state = PCG_REQ_CANCELLED;   // leaves its batch, and frees its budget, at the next tick
        return PCG_OK;
    case PCG_REQ_DONE:
        return fail(s->ctx, PCG_ERR_INVALID, "request " + std::to_string(id) + " has already finished");
    default:
        return PCG_OK;   // cancelled already
    }
}

pcg_status pcg_serve_placement(pcg_server* s, uint64_t id, int* ctx_index)
{
    if (!s || !ctx_index) return PCG_ERR_INVALID;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return PCG_ERR_NOT_FOUND;
    *ctx_index = it->second->lane;
    return PCG_OK;
}

pcg_status pcg_serve_state(pcg_server* s, uint64_t id, int* state)
{
    if (!s || !state) return PCG_ERR_INVALID;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return PCG_ERR_NOT_FOUND;
    *state = it->second->state;
    return PCG_OK;
}

pcg_status pcg_serve_fetch(pcg_server* s, uint64_t id, float* density, size_t n_floats, float* soa, uint32_t soa_max)
{
    if (!s) return PCG_ERR_INVALID;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return PCG_ERR_NOT_FOUND;
    Request* r = it->second.get();
    if (r->state == PCG_REQ_CANCELLED) return fail(s->ctx, PCG_ERR_INVALID, "request was cancelled");
    if (r->state != PCG_REQ_DONE) return PCG_ERR_NOT_READY;
    if (density) {
        if (n_floats != r->out_dens.size()) return fail(s->ctx, PCG_ERR_INVALID, "density size mismatch");
        std::memcpy(density, r->out_dens.data(), n_floats * sizeof(float));
    }
    if (soa && r->desc.n_cells) {
        if (soa_max < r->desc.n_cells) return fail(s->ctx, PCG_ERR_INVALID, "soa_max_cells < n_cells");
        for (int f = 0; f < NUM_FIELDS; ++f)
            std::memcpy(soa + static_cast<size_t>(f) * soa_max,
                        r->out_soa.data() + static_cast<size_t>(f) * r->desc.n_cells, r->desc.n_cells * sizeof(float));
    }
    return PCG_OK;
}

pcg_status pcg_serve_request_times(pcg_server* s, uint64_t id, double* submit_to_done, double* admit_to_done)
{
    if (!s) return PCG_ERR_INVALID;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return PCG_ERR_NOT_FOUND;
    Request* r = it->second.get();
    if (r->state == PCG_REQ_CANCELLED) return fail(s->ctx, PCG_ERR_INVALID, "request was cancelled");
    if (r->state != PCG_REQ_DONE) return PCG_ERR_NOT_READY;
    if (submit_to_done) *submit_to_done = r->t_done - r->t_submit;
    if (admit_to_done) *admit_to_done = r->t_done - r->t_admit;
    return PCG_OK;
}

pcg_status pcg_serve_totals(pcg_server* s, uint64_t* voxel_steps, uint64_t* cell_steps, uint64_t* bytes)
{
    if (!s) return PCG_ERR_INVALID;
    if (voxel_steps) *voxel_steps = s->voxel_steps;
    if (cell_steps) *cell_steps = s->cell_steps;
    if (bytes) {
        *bytes = 0;
        for (auto& L : s->lanes) *bytes += L->bytes_in_use;
    }
    return PCG_OK;
}

}  // extern "C"
