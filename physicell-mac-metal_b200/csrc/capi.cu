// capi.cu — the extern "C" entry points of include/pcg.h.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "capi.h"

using namespace pcg;


namespace {

thread_local std::string g_create_err;

int bad(pcg_ctx* ctx, const char* msg) { return fail(ctx, PCG_ERR_INVALID, msg); }

bool same_bytes(const void* a, const void* b, size_t n) { return std::memcmp(a, b, n) == 0; }

// Attach the diffusion grid of 'me' to the single instance of 'cells'.
int bind_me(pcg_cells* cells, const pcg_me* me)
{
    CellInst ci = cells->c.h_inst[0];
    fill_diff_inst(ci, me->d.inst[0]);
    if (!same_bytes(&ci, &cells->c.h_inst[0], sizeof ci)) {
        const CellInst& old = cells->c.h_inst[0];
        if (old.dx != ci.dx || old.dy != ci.dy || old.dz != ci.dz) cells->c.coef_dirty = true;
        cells->c.h_inst[0] = ci;
        cells->c.inst_dirty = true;
        cells->c.order_dirty = true;
    }
    cells->bound_me = me;
    return PCG_OK;
}

int bind_mech(pcg_cells* cells, const pcg_mech* mech)
{
    CellInst ci = cells->c.h_inst[0];
    fill_mech_inst(ci, mech->p, mech->ox, mech->oy, mech->oz);
    ci.mvox_base = 0;
    if (!same_bytes(&ci, &cells->c.h_inst[0], sizeof ci)) {
        cells->c.h_inst[0] = ci;
        cells->c.inst_dirty = true;
    }
    cells->bound_mech = mech;
    return PCG_OK;
}

int check_grid(pcg_ctx* ctx, const pcg_grid_params* g, const pcg_substrate_params* subs)
{
    if (!g) return bad(ctx, "grid is NULL");
    if (g->nx == 0 || g->ny == 0 || g->nz == 0) return bad(ctx, "grid dimensions must be >= 1");
    if (g->n_substrates > 0 && !subs) return bad(ctx, "substrates is NULL");
    if (!(g->dx > 0.f) || !(g->dy > 0.f) || !(g->dz > 0.f)) return bad(ctx, "voxel sizes must be > 0");
    if (!(g->dt >= 0.f)) return bad(ctx, "dt must be >= 0");
    return PCG_OK;
}

int check_mech(pcg_ctx* ctx, const pcg_mechanics_params* p)
{
    if (!p) return bad(ctx, "mechanics params is NULL");
    if (p->mech_grid_nx == 0 || p->mech_grid_ny == 0 || p->mech_grid_nz == 0)
        return bad(ctx, "mechanics grid dimensions must be >= 1");
    if (!(p->mechanics_voxel_size > 0.f)) return bad(ctx, "mechanics voxel size must be > 0");
    const uint64_t v = static_cast<uint64_t>(p->mech_grid_nx) * p->mech_grid_ny * p->mech_grid_nz;
    if (v >= 0xFFFFFFF0ull) return bad(ctx, "mechanics grid too large");
    return PCG_OK;
}

// Frees the context once nothing refers to it any more.
void ctx_free(pcg_ctx* ctx)
{
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (cudaStream_t c : {ctx->h2d, ctx->d2h})
        if (c) {
            cudaStreamSynchronize(c);
            cudaStreamDestroy(c);
        }
    for (cudaEvent_t e : ctx->copy_ev)
        if (e) cudaEventDestroy(e);
    for (cudaStream_t f : ctx->fork_st)
        if (f) {
            cudaStreamSynchronize(f);
            cudaStreamDestroy(f);
        }
    for (cudaEvent_t e : ctx->fork_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->status) cudaFree(ctx->status);
    delete ctx;
}

}  // namespace

namespace pcg {

void ctx_retain(pcg_ctx* ctx) { ctx->refs.fetch_add(1, std::memory_order_relaxed); }

void ctx_release(pcg_ctx* ctx)
{
    if (ctx->refs.fetch_sub(1, std::memory_order_acq_rel) == 1) ctx_free(ctx);
}

}  // namespace pcg

extern "C" {

int pcg_abi_version(void) { return PCG_ABI_VERSION; }

// ------------------------------------------------------------------ context

static pcg_status create_ctx(int device, void* stream, pcg_ctx** out)
{
    if (!out) return PCG_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        g_create_err = "no CUDA device";
        return PCG_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) {
        g_create_err = "device index out of range";
        return PCG_ERR_INVALID;
    }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        g_create_err = cudaGetErrorString(e);
        return PCG_ERR_CUDA;
    }
    pcg_ctx* c = new (std::nothrow) pcg_ctx();
    if (!c) return PCG_ERR_OOM;
    c->device = device;
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&c->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (stream) {
        c->stream = static_cast<cudaStream_t>(stream);
        c->own_stream = false;
    } else {
        e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            g_create_err = cudaGetErrorString(e);
            delete c;
            return PCG_ERR_CUDA;
        }
        c->own_stream = true;
    }
    // [0] the status word, [1] test switches (PCG_DEV_TEST_*)
    if (cudaMalloc(&c->status, 2 * sizeof(unsigned)) != cudaSuccess ||
        cudaMemsetAsync(c->status, 0, 2 * sizeof(unsigned), c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
        g_create_err = "status word allocation failed";
        if (c->own_stream) cudaStreamDestroy(c->stream);
        delete c;
        return PCG_ERR_OOM;
    }
    *out = c;
    return PCG_OK;
}

pcg_status pcg_create(int device, pcg_ctx** out) { return create_ctx(device, nullptr, out); }

pcg_status pcg_create_on_stream(int device, void* stream, pcg_ctx** out) { return create_ctx(device, stream, out); }

pcg_status pcg_destroy(pcg_ctx* ctx)
{
    if (ctx) pcg::ctx_release(ctx);
    return PCG_OK;
}

pcg_status pcg_join(pcg_ctx* ctx)
{
    if (!ctx) return PCG_ERR_INVALID;
    const cudaStream_t cs[2] = {ctx->h2d, ctx->d2h};
    for (int q = 0; q < 2; ++q) {
        if (!cs[q]) continue;
        PCG_CU(ctx, cudaEventRecord(ctx->copy_ev[q], cs[q]));
        PCG_CU(ctx, cudaStreamWaitEvent(ctx->stream, ctx->copy_ev[q], 0));
    }
    return PCG_OK;
}

pcg_status pcg_sync(pcg_ctx* ctx)
{
    if (!ctx) return PCG_ERR_INVALID;
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    for (cudaStream_t c : {ctx->h2d, ctx->d2h})
        if (c) PCG_CU(ctx, cudaStreamSynchronize(c));
    unsigned st = 0;
    PCG_CU(ctx, cudaMemcpy(&st, ctx->status, sizeof st, cudaMemcpyDeviceToHost));
    if (st) {
        PCG_CU(ctx, cudaMemsetAsync(ctx->status, 0, sizeof st, ctx->stream));
        PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
        return fail(ctx, PCG_ERR_DEVICE, std::string("a kernel stopped early:") + ((st & PCG_DEV_TIMEOUT) ? " wait limit reached" : "") +
                                              ((st & PCG_DEV_ALIGN) ? " unaligned bulk copy refused" : ""));
    }
    return PCG_OK;
}

void* pcg_stream(pcg_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

const char* pcg_last_error_string(const pcg_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_err.c_str(); }

uint64_t pcg_kernel_launches(const pcg_ctx* ctx) { return ctx ? ctx->launches : 0; }

uint32_t pcg_neighbor_hash(uint32_t cell) { return neighbor_hash_host(cell); }

pcg_status pcg_host_alloc(size_t bytes, void** out)
{
    if (!out) return PCG_ERR_INVALID;
    *out = nullptr;
    if (bytes == 0) return PCG_OK;
    return cudaMallocHost(out, bytes) == cudaSuccess ? PCG_OK : PCG_ERR_OOM;
}

pcg_status pcg_host_free(void* p)
{
    if (p) cudaFreeHost(p);
    return PCG_OK;
}

// ------------------------------------------------------------------ microenvironment

pcg_status pcg_me_create(pcg_ctx* ctx, const pcg_grid_params* grid, const pcg_substrate_params* subs, pcg_me** out)
{
    if (!ctx || !out) return PCG_ERR_INVALID;
    AllocStream pool_scope(ctx->stream);
    *out = nullptr;
    PCG_TRY(check_grid(ctx, grid, subs));
    pcg_me* me = new (std::nothrow) pcg_me();
    if (!me) return PCG_ERR_OOM;
    me->ctx = ctx;
    DiffInstance di;
    di.g = *grid;
    di.subs.assign(subs, subs + grid->n_substrates);
    std::vector<DiffInstance> v{di};
    int rc = me->d.build(ctx, std::move(v));
    if (rc != PCG_OK) {
        delete me;
        return rc;
    }
    ctx_retain(ctx);
    *out = me;
    return PCG_OK;
}

pcg_status pcg_me_destroy(pcg_me* me)
{
    if (!me) return PCG_OK;
    pcg_ctx* ctx = me->ctx;
    delete me;
    ctx_release(ctx);
    return PCG_OK;
}

pcg_status pcg_me_fill(pcg_me* me, const float* v)
{
    if (!me || !v) return PCG_ERR_INVALID;
    return me->d.fill(0, v);
}

pcg_status pcg_me_upload(pcg_me* me, const float* host, size_t n)
{
    if (!me || !host) return PCG_ERR_INVALID;
    if (n != me->d.total_vox_sub) return bad(me->ctx, "density size mismatch");
    return me->d.upload(0, host);
}

pcg_status pcg_me_download(pcg_me* me, float* host, size_t n)
{
    if (!me || !host) return PCG_ERR_INVALID;
    if (n != me->d.total_vox_sub) return bad(me->ctx, "density size mismatch");
    return me->d.download(0, host);
}

pcg_status pcg_me_diffuse(pcg_me* me, int n_steps)
{
    if (!me || n_steps < 0) return PCG_ERR_INVALID;
    for (int s = 0; s < n_steps; ++s) PCG_TRY(me->d.sweeps(false, nullptr));
    return PCG_OK;
}

pcg_status pcg_me_apply_dirichlet(pcg_me* me)
{
    if (!me) return PCG_ERR_INVALID;
    return me->d.dirichlet();
}

pcg_status pcg_me_secrete(pcg_me* me, pcg_cells* cells, double dt)
{
    if (!me || !cells) return PCG_ERR_INVALID;
    if (cells->S != me->d.inst[0].g.n_substrates) return bad(me->ctx, "cells and microenvironment substrate counts differ");
    if (cells->c.n == 0) return PCG_OK;
    PCG_TRY(bind_me(cells, me));
    PCG_TRY(cells->c.prepare_secretion(dt, me->d.total_vox));
    return cells->c.secrete(me->d, nullptr);
}

pcg_status pcg_me_step(pcg_me* me, pcg_cells* cells, int n_steps)
{
    if (!me || n_steps < 0) return PCG_ERR_INVALID;
    const bool sec = cells && cells->c.n > 0;
    if (sec) {
        if (cells->S != me->d.inst[0].g.n_substrates)
            return bad(me->ctx, "cells and microenvironment substrate counts differ");
        PCG_TRY(bind_me(cells, me));
    }
    const double dt = me->d.inst[0].g.dt;
    for (int s = 0; s < n_steps; ++s) {
        PCG_TRY(me->d.sweeps(true, nullptr));
        if (sec) {
            PCG_TRY(cells->c.prepare_secretion(dt, me->d.total_vox));
            PCG_TRY(cells->c.secrete(me->d, nullptr));
        }
    }
    return PCG_OK;
}

pcg_status pcg_me_gradients(pcg_me* me, float* gx, float* gy, float* gz, size_t n)
{
    if (!me) return PCG_ERR_INVALID;
    if (n != me->d.total_vox_sub) return bad(me->ctx, "gradient size mismatch");
    AllocStream pool_scope(me->ctx->stream);
    DevBuf buf;
    PCG_CU(me->ctx, buf.alloc(3 * n * sizeof(float) + 16));
    float* b = buf.as<float>();
    PCG_TRY(me->d.gradients(gx ? b : nullptr, gy ? b + n : nullptr, gz ? b + 2 * n : nullptr));
    float* outs[3] = {gx, gy, gz};
    for (int q = 0; q < 3; ++q)
        if (outs[q])
            PCG_CU(me->ctx, cudaMemcpyAsync(outs[q], b + q * n, n * sizeof(float), cudaMemcpyDeviceToHost, me->ctx->stream));
    PCG_CU(me->ctx, cudaStreamSynchronize(me->ctx->stream));
    return PCG_OK;
}

pcg_status pcg_me_device_density(pcg_me* me, float** dptr, size_t* row_pitch, size_t* substrate_pitch)
{
    if (!me) return PCG_ERR_INVALID;
    if (dptr) *dptr = me->d.dens.as<float>();
    if (row_pitch) *row_pitch = me->d.inst[0].px;
    if (substrate_pitch) *substrate_pitch = me->d.inst[0].pitch;
    return PCG_OK;
}

// ------------------------------------------------------------------ cells

pcg_status pcg_cells_create(pcg_ctx* ctx, uint32_t max_cells, uint32_t S, pcg_cells** out)
{
    if (!ctx || !out) return PCG_ERR_INVALID;
    AllocStream pool_scope(ctx->stream);
    *out = nullptr;
    if (max_cells == 0) return bad(ctx, "max_cells must be >= 1");
    pcg_cells* c = new (std::nothrow) pcg_cells();
    if (!c) return PCG_ERR_OOM;
    c->ctx = ctx;
    c->S = S;
    const uint64_t rc = static_cast<uint64_t>(max_cells) * std::max<uint32_t>(S, 1);
    if (rc > 0xFFFFFFFFull) {
        delete c;
        return bad(ctx, "max_cells * substrates exceeds 2^32");
    }
    int r = c->c.create(ctx, max_cells, static_cast<uint32_t>(rc), 1);
    if (r == PCG_OK) r = c->c.set_active(0, max_cells, nullptr);
    if (r != PCG_OK) {
        delete c;
        return r;
    }
    c->c.has_active = false;
    c->c.h_inst[0].S = S;
    ctx_retain(ctx);
    *out = c;
    return PCG_OK;
}

pcg_status pcg_cells_destroy(pcg_cells* c)
{
    if (!c) return PCG_OK;
    pcg_ctx* ctx = c->ctx;
    delete c;
    ctx_release(ctx);
    return PCG_OK;
}

pcg_status pcg_cells_upload(pcg_cells* c, const float* soa, uint32_t n, uint32_t soa_max)
{
    if (!c || (!soa && n)) return PCG_ERR_INVALID;
    if (n > c->c.max_cells) return bad(c->ctx, "n_cells exceeds max_cells");
    if (soa_max < n) return bad(c->ctx, "soa_max_cells < n_cells");
    c->c.n = n;
    if (c->c.h_inst[0].n_cells != n) {
        c->c.h_inst[0].n_cells = n;
        c->c.inst_dirty = true;
    }
    PCG_TRY(c->c.upload_soa(0, n, soa, soa_max, 0, NUM_FIELDS));
    c->c.coef_dirty = c->c.order_dirty = true;
    PCG_CU(c->ctx, cudaStreamSynchronize(c->ctx->stream));
    return PCG_OK;
}

pcg_status pcg_cells_download(pcg_cells* c, float* soa, uint32_t soa_max)
{
    if (!c || !soa) return PCG_ERR_INVALID;
    if (soa_max < c->c.n) return bad(c->ctx, "soa_max_cells < n_cells");
    PCG_TRY(c->c.download_soa(0, c->c.n, soa, soa_max, 0, NUM_FIELDS));
    PCG_CU(c->ctx, cudaStreamSynchronize(c->ctx->stream));
    return PCG_OK;
}

pcg_status pcg_cells_upload_fields(pcg_cells* c, uint32_t first, uint32_t count, const float* soa, uint32_t soa_max)
{
    if (!c || !soa || first + count > NUM_FIELDS || first + count < first) return PCG_ERR_INVALID;
    if (soa_max < c->c.n) return bad(c->ctx, "soa_max_cells < n_cells");
    PCG_TRY(c->c.upload_soa(0, c->c.n, soa, soa_max, first, count));
    PCG_CU(c->ctx, cudaStreamSynchronize(c->ctx->stream));
    return PCG_OK;
}

pcg_status pcg_cells_download_fields(pcg_cells* c, uint32_t first, uint32_t count, float* soa, uint32_t soa_max)
{
    if (!c || !soa || first + count > NUM_FIELDS || first + count < first) return PCG_ERR_INVALID;
    if (soa_max < c->c.n) return bad(c->ctx, "soa_max_cells < n_cells");
    PCG_TRY(c->c.download_soa(0, c->c.n, soa, soa_max, first, count));
    PCG_CU(c->ctx, cudaStreamSynchronize(c->ctx->stream));
    return PCG_OK;
}

pcg_status pcg_cells_set_secretion(pcg_cells* c, const double* sec, const double* upt, const double* sat,
                                   const double* ne, const uint8_t* active)
{
    if (!c) return PCG_ERR_INVALID;
    const uint32_t count = c->c.n * c->S;
    PCG_TRY(c->c.set_rates(0, count, sec, upt, sat, ne));
    PCG_TRY(c->c.set_active(0, c->c.n, active));
    if (!active) c->c.has_active = false;
    return PCG_OK;
}

pcg_status pcg_cells_download_secretion(pcg_cells* c, double* sec, double* upt, double* sat, double* ne,
                                        uint8_t* active)
{
    if (!c) return PCG_ERR_INVALID;
    const size_t cap = c->c.rates.bytes / (4 * sizeof(double));
    const size_t count = static_cast<size_t>(c->c.n) * c->S;
    double* dst[4] = {sec, upt, sat, ne};
    for (int q = 0; q < 4; ++q)
        if (dst[q] && count)
            PCG_CU(c->ctx, cudaMemcpyAsync(dst[q], c->c.rates.as<double>() + q * cap, count * sizeof(double),
                                           cudaMemcpyDeviceToHost, c->ctx->stream));
    if (active && c->c.n)
        PCG_CU(c->ctx, cudaMemcpyAsync(active, c->c.active.p, c->c.n, cudaMemcpyDeviceToHost, c->ctx->stream));
    PCG_CU(c->ctx, cudaStreamSynchronize(c->ctx->stream));
    return PCG_OK;
}

pcg_status pcg_removal_plan(uint32_t n_cells, const uint32_t* indices, uint32_t count, uint32_t* dest, uint32_t* src,
                            uint32_t* n_moves, uint32_t* n_final)
{
    if ((!indices && count) || !n_moves || !n_final || ((!dest || !src) && count)) return PCG_ERR_INVALID;
    std::vector<uint2> moves;
    *n_final = removal_plan(n_cells, indices, count, &moves);
    *n_moves = static_cast<uint32_t>(moves.size());
    for (size_t k = 0; k < moves.size(); ++k) {
        dest[k] = moves[k].x;
        src[k] = moves[k].y;
    }
    return PCG_OK;
}

pcg_status pcg_cells_remove(pcg_cells* c, const uint32_t* indices, uint32_t count)
{
    if (!c || (!indices && count)) return PCG_ERR_INVALID;
    AllocStream pool_scope(c->ctx->stream);
    std::vector<uint2> moves;
    const uint32_t n = removal_plan(c->c.n, indices, count, &moves);
    if (!moves.empty()) {
        DevBuf dm;
        PCG_CU(c->ctx, dm.alloc(moves.size() * sizeof(uint2)));
        PCG_CU(c->ctx, cudaMemcpyAsync(dm.p, moves.data(), moves.size() * sizeof(uint2), cudaMemcpyHostToDevice,
                                       c->ctx->stream));
        const uint64_t rate_cap = c->c.rates.bytes / (4 * sizeof(double));
        PCG_CU(c->ctx, launch_cells_move(c->ctx->stream, c->c.soa.as<float>(), c->c.max_cells, dm.as<uint2>(),
                                         static_cast<uint32_t>(moves.size()), c->c.rates.as<double>(), rate_cap, c->S,
                                         c->c.active.as<uint8_t>(), c->c.pos64.as<double>()));
        c->ctx->launches++;
        PCG_CU(c->ctx, cudaStreamSynchronize(c->ctx->stream));   // the move list is released on return
    }
    if (n != c->c.n) {
        c->c.n = n;
        c->c.h_inst[0].n_cells = n;
        c->c.inst_dirty = true;
        c->c.coef_dirty = c->c.order_dirty = true;
    }
    return PCG_OK;
}

pcg_status pcg_cells_append(pcg_cells* c, const float* soa, uint32_t count, uint32_t soa_max, const double* sec,
                            const double* upt, const double* sat, const double* ne, const uint8_t* active)
{
    if (!c || (!soa && count)) return PCG_ERR_INVALID;
    if (count == 0) return PCG_OK;
    if (soa_max < count) return bad(c->ctx, "soa_max_cells < count");
    if (static_cast<uint64_t>(c->c.n) + count > c->c.max_cells) return bad(c->ctx, "appending past max_cells");
    const uint32_t n0 = c->c.n;
    PCG_TRY(c->c.upload_soa(n0, count, soa, soa_max, 0, NUM_FIELDS));
    PCG_TRY(c->c.clear_masters(n0, count));   // places past the count may hold removed cells' masters
    PCG_TRY(c->c.set_rates(n0 * c->S, count * c->S, sec, upt, sat, ne));
    PCG_TRY(c->c.set_active(n0, count, active));
    c->c.n = n0 + count;
    c->c.h_inst[0].n_cells = c->c.n;
    c->c.inst_dirty = true;
    c->c.coef_dirty = c->c.order_dirty = true;
    PCG_CU(c->ctx, cudaStreamSynchronize(c->ctx->stream));
    return PCG_OK;
}

pcg_status pcg_cells_download_positions64(pcg_cells* c, double* xyz, uint32_t n_cells)
{
    if (!c || (!xyz && n_cells)) return PCG_ERR_INVALID;
    if (n_cells != c->c.n) return bad(c->ctx, "n_cells must equal the current cell count");
    return c->c.download_positions(0, n_cells, xyz);
}

pcg_status pcg_cells_set_voxel_refresh(pcg_cells* c, const pcg_me* me, int on)
{
    if (!c || (on && !me)) return PCG_ERR_INVALID;
    if (on) PCG_TRY(bind_me(c, me));
    const uint32_t f = on ? (c->c.h_inst[0].flags | INST_REFRESH_VOXELS) : (c->c.h_inst[0].flags & ~INST_REFRESH_VOXELS);
    if (f != c->c.h_inst[0].flags) {
        c->c.h_inst[0].flags = f;
        c->c.inst_dirty = true;
    }
    return PCG_OK;
}

pcg_status pcg_cells_count(pcg_cells* c, uint32_t* n)
{
    if (!c || !n) return PCG_ERR_INVALID;
    *n = c->c.n;
    return PCG_OK;
}

pcg_status pcg_cells_device_soa(pcg_cells* c, float** dptr, uint32_t* max_cells)
{
    if (!c) return PCG_ERR_INVALID;
    if (dptr) *dptr = c->c.soa.as<float>();
    if (max_cells) *max_cells = c->c.max_cells;
    return PCG_OK;
}

// ------------------------------------------------------------------ mechanics

pcg_status pcg_mech_create(pcg_ctx* ctx, const pcg_mechanics_params* p, float x_min, float y_min, float z_min,
                           uint32_t max_cells, pcg_mech** out)
{
    if (!ctx || !out) return PCG_ERR_INVALID;
    AllocStream pool_scope(ctx->stream);
    *out = nullptr;
    PCG_TRY(check_mech(ctx, p));
    pcg_mech* m = new (std::nothrow) pcg_mech();
    if (!m) return PCG_ERR_OOM;
    m->ctx = ctx;
    m->p = *p;
    m->ox = x_min;
    m->oy = y_min;
    m->oz = z_min;
    const uint32_t V = p->mech_grid_nx * p->mech_grid_ny * p->mech_grid_nz;
    int rc = m->m.create(ctx, V, max_cells);
    if (rc != PCG_OK) {
        delete m;
        return rc;
    }
    ctx_retain(ctx);
    *out = m;
    return PCG_OK;
}

pcg_status pcg_mech_destroy(pcg_mech* m)
{
    if (!m) return PCG_OK;
    pcg_ctx* ctx = m->ctx;
    delete m;
    ctx_release(ctx);
    return PCG_OK;
}

pcg_status pcg_mech_forces(pcg_mech* m, pcg_cells* c)
{
    if (!m || !c) return PCG_ERR_INVALID;
    if (c->c.n > m->m.cap) return bad(m->ctx, "more cells than the mechanics object was created for");
    PCG_TRY(bind_mech(c, m));
    return m->m.forces(c->c, nullptr);
}

pcg_status pcg_mech_integrate(pcg_mech* m, pcg_cells* c, float dt)
{
    if (!m || !c || !(dt >= 0.f)) return PCG_ERR_INVALID;
    PCG_TRY(bind_mech(c, m));
    return m->m.integrate(c->c, dt, nullptr);
}

pcg_status pcg_mech_update(pcg_mech* m, pcg_cells* c, float dt)
{
    PCG_TRY(pcg_mech_forces(m, c));
    return pcg_mech_integrate(m, c, dt);
}

pcg_status pcg_mech_bins(pcg_mech* m, uint32_t* start, uint32_t* sorted)
{
    if (!m) return PCG_ERR_INVALID;
    pcg_ctx* ctx = m->ctx;
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    if (start)
        PCG_CU(ctx, cudaMemcpy(start, m->m.start.p, (static_cast<size_t>(m->m.total_mvox) + 1) * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost));
    if (sorted) {
        uint32_t n = 0;
        PCG_CU(ctx, cudaMemcpy(&n, m->m.start.as<uint32_t>() + m->m.total_mvox, sizeof n, cudaMemcpyDeviceToHost));
        if (n) PCG_CU(ctx, cudaMemcpy(sorted, m->m.sorder.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    }
    return PCG_OK;
}

uint32_t pcg_mech_total_voxels(const pcg_mech* m) { return m ? m->m.total_mvox : 0; }

pcg_status pcg_mech_set_diagnostics(pcg_mech* m, int on)
{
    if (!m) return PCG_ERR_INVALID;
    m->m.diag = on != 0;
    return PCG_OK;
}

pcg_status pcg_mech_neighbor_stats(pcg_mech* m, uint32_t* count, uint32_t* hash)
{
    if (!m) return PCG_ERR_INVALID;
    if (!m->m.diag) return bad(m->ctx, "diagnostics are off");
    pcg_ctx* ctx = m->ctx;
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    uint32_t n = 0;
    PCG_CU(ctx, cudaMemcpy(&n, m->m.start.as<uint32_t>() + m->m.total_mvox, sizeof n, cudaMemcpyDeviceToHost));
    if (count && n) PCG_CU(ctx, cudaMemcpy(count, m->m.dcnt.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (hash && n) PCG_CU(ctx, cudaMemcpy(hash, m->m.dhash.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return PCG_OK;
}

void pcg_debug_alloc_stats(uint64_t* device_mallocs, uint64_t* pool_reuses)
{
    alloc_stats(device_mallocs, pool_reuses);
}

void pcg_debug_fail_alloc(uint64_t nth) { fail_alloc_after(nth); }

pcg_status pcg_debug_give_up_waits(pcg_ctx* ctx, int on)
{
    if (!ctx) return PCG_ERR_INVALID;
    const unsigned v = on ? PCG_DEV_TEST_GIVE_UP : 0u;
    PCG_CU(ctx, cudaMemcpyAsync(ctx->status + 1, &v, sizeof v, cudaMemcpyHostToDevice, ctx->stream));
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return PCG_OK;
}

}  // extern "C"
