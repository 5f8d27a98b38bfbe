// batch.cu — many independent simulations advanced together.
//
// All instances share one density arena, one cell SoA and one mechanics
// key space; every phase of a main-loop sub-step is one persistent kernel
// over a flat work list of all instances (src/main.mm:341-391 ordering:
// sweeps -> Dirichlet reset (fused) -> secretion -> [mechanics]).  The
// sub-step with and without mechanics, and a whole mechanics period, are
// each captured once into a CUDA graph, so one sub-step, or one period
// where a call covers it, is one graph launch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "batch.h"

using namespace pcg;

namespace pcg {

uint64_t instance_bytes(const pcg_instance_desc& d)
{
    const uint64_t nv = static_cast<uint64_t>(d.grid.nx) * d.grid.ny * d.grid.nz;
    const uint64_t S = d.grid.n_substrates;
    const uint64_t pitch = (nv + 31) / 32 * 32;
    const uint64_t n = d.n_cells;
    const uint64_t V = static_cast<uint64_t>(d.mech.mech_grid_nx) * d.mech.mech_grid_ny * d.mech.mech_grid_nz;
    uint64_t b = pitch * S * 4;                            // density
    b += (nv / 32 + 3) * 32 * S;                           // tile lists (~32 B per 32 lines per axis)
    b += n * (NUM_FIELDS * 4 + 4 + 1);                     // SoA, instance id, active
    b += n * 3 * 8;                                        // FP64 master positions
    b += n * S * (4 * 8 + 3 * 8 * 2);                      // rates, secretion constants (cell and sorted order)
    b += n * 4 * 6 * 2;                                    // two sort workspaces
    b += n * 8;                                            // per-run word (instance, density element)
    b += n * (16 + 16 + 8);                                // sorted SoA, diagnostics
    b += (V + 1) * 4 * 2;                                  // counts, start
    b += (n / 2048 + 2) * (257 * 4 + sizeof(SegTile) + 8) + 4096;   // sort tiles, digit rows, run scan
    return b;
}

int Batch::create(pcg_ctx* c, const pcg_instance_desc* descs, uint32_t n, const pcg_batch_options* opt,
                  const std::vector<DevSource>* src, bool masked_steps)
{
    ctx = c;
    masked = masked_steps;
    AllocStream pool_scope(ctx->stream);   // buffers come from (and return to) the device pool
    auto from = [&](uint32_t i) -> const DevSource* {
        return (src && i < src->size() && (*src)[i].batch) ? &(*src)[i] : nullptr;
    };
    if (n == 0) return fail(ctx, PCG_ERR_INVALID, "no instances");
    use_graphs = opt ? opt->use_graphs != 0 : true;
    profile = opt ? opt->profile_phases != 0 : false;
    const bool tune = opt ? opt->autotune != 0 : true;
    if (opt && opt->tune_cache) tune_cache = opt->tune_cache;
    dt_diff = descs[0].grid.dt;
    dt_mech = descs[0].dt_mechanics > 0.f ? descs[0].dt_mechanics : descs[0].mech.dt;
    std::vector<DiffInstance> di(n);
    uint64_t cells_total = 0, rates_total = 0, mvox_total = 0;
    ncell.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        const pcg_instance_desc& d = descs[i];
        const float dm = d.dt_mechanics > 0.f ? d.dt_mechanics : d.mech.dt;
        if (d.grid.dt != descs[0].grid.dt || dm != dt_mech)
            return fail(ctx, PCG_ERR_INVALID, "instances of one batch must share dt_diffusion and dt_mechanics");
        if (d.grid.n_substrates > 0 && !d.substrates) return fail(ctx, PCG_ERR_INVALID, "substrates is NULL");
        if (d.n_cells > 0 && !from(i) && (!d.cells_soa || d.cells_soa_max < d.n_cells))
            return fail(ctx, PCG_ERR_INVALID, "cells_soa missing or cells_soa_max < n_cells");
        if (d.mech.mech_grid_nx == 0 || d.mech.mech_grid_ny == 0 || d.mech.mech_grid_nz == 0 ||
            !(d.mech.mechanics_voxel_size > 0.f))
            return fail(ctx, PCG_ERR_INVALID, "bad mechanics grid");
        di[i].g = d.grid;
        di[i].subs.assign(d.substrates, d.substrates + d.grid.n_substrates);
        ncell[i] = d.n_cells;
        cells_total += d.n_cells;
        rates_total += static_cast<uint64_t>(d.n_cells) * d.grid.n_substrates;
        mvox_total += static_cast<uint64_t>(d.mech.mech_grid_nx) * d.mech.mech_grid_ny * d.mech.mech_grid_nz;
    }
    if (cells_total > 0xFFFFFFF0ull || rates_total > 0xFFFFFFF0ull || mvox_total > 0xFFFFFFF0ull)
        return fail(ctx, PCG_ERR_INVALID, "batch too large for 32-bit indices");
    d.use_planes = !(opt && opt->disable_planes);
    PCG_TRY(d.build(ctx, std::move(di)));
    for (uint32_t i = 0; i < n; ++i) {
        if (const DevSource* ds = from(i)) {
            const DiffInstance& so = ds->batch->d.inst[ds->index];
            const DiffInstance& de = d.inst[i];
            if (so.nvox() != de.nvox() || so.g.n_substrates != de.g.n_substrates)
                return fail(ctx, PCG_ERR_INVALID, "device source does not match the instance");
            for (uint32_t s = 0; s < de.g.n_substrates; ++s)
                PCG_CU(ctx, cudaMemcpyAsync(d.dens.as<float>() + de.dens_off + s * de.pitch,
                                            ds->batch->d.dens.as<float>() + so.dens_off + s * so.pitch,
                                            de.rows() * de.px * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
        } else if (descs[i].initial_density) {
            PCG_TRY(d.upload(i, descs[i].initial_density));
        } else if (descs[i].initial_values) {
            PCG_TRY(d.fill(i, descs[i].initial_values));
        }
    }
    // cells.  A server rebuilds its batch whenever requests come and go:
    // its cell arrays get power-of-two capacities, so consecutive rebuilds
    // ask the device pool for the same sizes and find the freed blocks.
    auto capacity = [&](uint64_t v) {
        v = std::max<uint64_t>(v, 1);
        if (!masked) return v;
        uint64_t c = 1;
        while (c < v) c <<= 1;
        return std::min<uint64_t>(c, 0xFFFFFFF0ull);
    };
    const uint32_t cell_cap = static_cast<uint32_t>(capacity(cells_total));
    PCG_TRY(c_.create(ctx, cell_cap, static_cast<uint32_t>(capacity(rates_total)), n));
    c_.n = static_cast<uint32_t>(cells_total);
    c_.n_rate = static_cast<uint32_t>(rates_total);
    PCG_TRY(c_.set_cell_instances(ncell));
    uint32_t coff = 0, roff = 0, moff = 0;
    any_refresh = false;
    for (uint32_t i = 0; i < n; ++i) {
        const pcg_instance_desc& ds = descs[i];
        CellInst& ci = c_.h_inst[i];
        ci = CellInst{};
        fill_diff_inst(ci, d.inst[i]);
        fill_mech_inst(ci, ds.mech, ds.grid.x_min, ds.grid.y_min, ds.grid.z_min);
        ci.dt_mech = dt_mech;
        ci.cell_off = coff;
        ci.n_cells = ds.n_cells;
        ci.rate_off = roff;
        ci.mvox_base = moff;
        ci.flags = (ds.flags & PCG_INST_REFRESH_VOXELS) ? INST_REFRESH_VOXELS : 0u;
        any_refresh = any_refresh || ci.flags;
        if (ds.n_cells && from(i)) {
            const Batch& sb = *from(i)->batch;
            const CellInst& so = sb.c_.h_inst[from(i)->index];
            if (so.n_cells != ds.n_cells || so.S != ds.grid.n_substrates)
                return fail(ctx, PCG_ERR_INVALID, "device source cells do not match the instance");
            PCG_CU(ctx, cudaMemcpy2DAsync(c_.soa.as<float>() + coff, static_cast<size_t>(c_.max_cells) * sizeof(float),
                                          sb.c_.soa.as<float>() + so.cell_off,
                                          static_cast<size_t>(sb.c_.max_cells) * sizeof(float),
                                          static_cast<size_t>(ds.n_cells) * sizeof(float), NUM_FIELDS,
                                          cudaMemcpyDeviceToDevice, ctx->stream));
            const size_t cap_new = c_.rates.bytes / (4 * sizeof(double));
            const size_t cap_old = sb.c_.rates.bytes / (4 * sizeof(double));
            const size_t nr = static_cast<size_t>(ds.n_cells) * ds.grid.n_substrates;
            for (int q = 0; q < 4; ++q)
                PCG_CU(ctx, cudaMemcpyAsync(c_.rates.as<double>() + q * cap_new + roff,
                                            sb.c_.rates.as<double>() + q * cap_old + so.rate_off, nr * sizeof(double),
                                            cudaMemcpyDeviceToDevice, ctx->stream));
            PCG_CU(ctx, cudaMemcpyAsync(c_.active.as<uint8_t>() + coff, sb.c_.active.as<uint8_t>() + so.cell_off,
                                        ds.n_cells, cudaMemcpyDeviceToDevice, ctx->stream));
            PCG_CU(ctx, cudaMemcpy2DAsync(c_.pos64.as<double>() + coff, static_cast<size_t>(c_.max_cells) * sizeof(double),
                                          sb.c_.pos64.as<double>() + so.cell_off,
                                          static_cast<size_t>(sb.c_.max_cells) * sizeof(double),
                                          static_cast<size_t>(ds.n_cells) * sizeof(double), 3,
                                          cudaMemcpyDeviceToDevice, ctx->stream));
            if (sb.c_.has_active) c_.has_active = true;
            c_.coef_dirty = c_.order_dirty = true;
        } else if (ds.n_cells) {
            PCG_TRY(c_.upload_soa(coff, ds.n_cells, ds.cells_soa, ds.cells_soa_max, 0, NUM_FIELDS));
            PCG_TRY(c_.set_rates(roff, ds.n_cells * ds.grid.n_substrates, ds.secretion, ds.uptake, ds.saturation,
                                 ds.net_export));
            PCG_TRY(c_.set_active(coff, ds.n_cells, ds.active));
            if (ds.active) c_.has_active = true;
        }
        coff += ds.n_cells;
        roff += ds.n_cells * ds.grid.n_substrates;
        moff += ds.mech.mech_grid_nx * ds.mech.mech_grid_ny * ds.mech.mech_grid_nz;
    }
    c_.inst_dirty = true;
    PCG_TRY(c_.sync_inst());
    PCG_TRY(m_.create(ctx, moff, cell_cap));
    m_.lazy_sorder = true;   // only pcg_batch_mech_bins reads the stable order
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    if (c_.n) PCG_TRY(c_.prepare_secretion(dt_diff, d.total_vox));
    if (tune) {
        if (!tune_cache.empty()) Tuner::get().load(tune_cache);
        PCG_TRY(d.tune());
    }
    if (opt) {
        PCG_TRY(d.pin(0, opt->pin_x));
        PCG_TRY(d.pin(1, opt->pin_cols));
    }
    PCG_TRY(tune_cells(opt, tune));
    if (tune && !tune_cache.empty()) Tuner::get().save(tune_cache);
    for (int q = 0; q < 8; ++q) PCG_CU(ctx, cudaEventCreate(&ev[q]));
    if (masked) {
        PCG_CU(ctx, mask_d.alloc(n));
        PCG_CU(ctx, cudaMemsetAsync(mask_d.p, STEP_DIFFUSE | STEP_MECH, n, ctx->stream));
    }
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    if (use_graphs) {
        PCG_TRY(capture(false, &g_diff, &launches_diff));
        PCG_TRY(capture(true, &g_mech, &launches_mech));
        // sub-steps from a reset accumulator to the firing one, as step() counts them
        double a = 0.0;
        int len = 0;
        for (bool fire = false; !fire && len <= kMaxPeriod; ++len) {
            a += dt_diff;
            fire = a >= dt_mech - 0.5 * dt_diff;
        }
        if (!masked && len >= 2 && len <= kMaxPeriod) {
            period_len = len;
            PCG_TRY(capture(true, &g_period, &launches_period, len - 1));
        }
    } else {
        launches_diff = count_launches(false);
        launches_mech = count_launches(true);
    }
    return PCG_OK;
}

Batch::~Batch()
{
    if (ctx && (stage_in.p || stage_cells.p || stage_dens.p)) {   // copies may still read or write them
        if (ctx->h2d) cudaStreamSynchronize(ctx->h2d);
        if (ctx->d2h) cudaStreamSynchronize(ctx->d2h);
        cudaStreamSynchronize(ctx->stream);
    }
    for (cudaEvent_t e : {ev_in_done, ev_in_used, ev_cells_ready, ev_cells_done, ev_dens_ready, ev_dens_done})
        if (e) cudaEventDestroy(e);
    for (cudaGraphExec_t g : {g_diff, g_mech, g_period})
        if (g) cudaGraphExecDestroy(g);
    for (int q = 0; q < 8; ++q)
        if (ev[q]) cudaEventDestroy(ev[q]);
}

namespace {

int log2_bucket(uint64_t v)
{
    int b = 0;
    while ((1ull << (b + 1)) <= v) ++b;
    return b;
}

bool valid_threads(int t, int hi) { return t >= 32 && t <= hi && t % 32 == 0; }

}  // namespace

int Batch::tune_cells(const pcg_batch_options* opt, bool tune)
{
    const int pin_f = opt ? opt->pin_forces : 0, pin_t = opt ? opt->pin_cell_threads : 0;
    if (pin_f) {
        const int t = pin_f / 1000, q = pin_f % 1000;
        if (!valid_threads(t, 256) || (q != 0 && q != 16 && q != 32 && q != 64))
            return fail(ctx, PCG_ERR_INVALID, "pin_forces must be threads (32..256, multiple of 32) * 1000 + queue (0, 16, 32, 64)");
        m_.fshape.block = t;
        m_.fshape.queue = q;
    }
    if (pin_t) {
        if (!valid_threads(pin_t, 256)) return fail(ctx, PCG_ERR_INVALID, "pin_cell_threads must be 32..256, a multiple of 32");
        c_.sec_block = m_.bin_block = m_.int_block = pin_t;
    }
    if (!tune || c_.n == 0 || (pin_f && pin_t)) return PCG_OK;
    const std::string sfx = ":c" + std::to_string(log2_bucket(c_.n)) + ":v" + std::to_string(log2_bucket(m_.total_mvox)) +
                            ":r" + std::to_string(log2_bucket(c_.n_rate));
    const std::string kf = "forces" + sfx, ks = "secrete" + sfx, kb = "bin" + sfx, ki = "integrate" + sfx;
    int vf = 0, vs = 0, vb = 0, vi = 0;
    Tuner& T = Tuner::get();
    const bool cached = T.lookup(kf, &vf) && T.lookup(ks, &vs) && T.lookup(kb, &vb) && T.lookup(ki, &vi);
    if (!cached) {
        // everything the timed launches write: the cell SoA, the master
        // positions and the density (secretion)
        DevBuf b_soa, b_pos, b_dens;
        if (b_soa.alloc(c_.soa.bytes) != cudaSuccess || b_pos.alloc(c_.pos64.bytes) != cudaSuccess ||
            b_dens.alloc(d.dens.bytes) != cudaSuccess) {
            cudaGetLastError();
            return PCG_OK;   // not enough memory to tune safely: keep the defaults
        }
        cudaStream_t st = ctx->stream;
        PCG_CU(ctx, cudaMemcpyAsync(b_soa.p, c_.soa.p, c_.soa.bytes, cudaMemcpyDeviceToDevice, st));
        PCG_CU(ctx, cudaMemcpyAsync(b_pos.p, c_.pos64.p, c_.pos64.bytes, cudaMemcpyDeviceToDevice, st));
        PCG_CU(ctx, cudaMemcpyAsync(b_dens.p, d.dens.p, d.dens.bytes, cudaMemcpyDeviceToDevice, st));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        PCG_CU(ctx, cudaEventCreate(&e0));
        PCG_CU(ctx, cudaEventCreate(&e1));
        const uint64_t launches0 = ctx->launches;
        const bool order_dirty = c_.order_dirty;   // the timed AB2 launches may flag it (voxel refresh)
        // best of the candidates by the time of 3 launches after a warm one
        auto pick = [&](const std::vector<int>& cands, auto set, auto run, int* best) -> int {
            float best_ms = 1e30f;
            for (int c : cands) {
                set(c);
                PCG_TRY(run());
                PCG_CU(ctx, cudaEventRecord(e0, st));
                for (int r = 0; r < 3; ++r) PCG_TRY(run());
                PCG_CU(ctx, cudaEventRecord(e1, st));
                PCG_CU(ctx, cudaEventSynchronize(e1));
                float ms = 0;
                PCG_CU(ctx, cudaEventElapsedTime(&ms, e0, e1));
                if (ms < best_ms) {
                    best_ms = ms;
                    *best = c;
                }
            }
            set(*best);
            return PCG_OK;
        };
        int rc = pick({128, 256, 512, 1024}, [&](int b) { m_.bin_block = b; },
                      [&]() { return m_.binsort(c_, nullptr); }, &vb);
        std::vector<int> fc;
        for (int t : {64, 128, 256})
            for (int q : {0, 16, 32, 64}) fc.push_back(t * 1000 + q);
        if (rc == PCG_OK)
            rc = pick(fc, [&](int v) { m_.fshape.block = v / 1000; m_.fshape.queue = v % 1000; },
                      [&]() { return m_.force_pass(c_, nullptr); }, &vf);
        if (rc == PCG_OK)
            rc = pick({64, 128, 256}, [&](int b) { c_.sec_block = b; }, [&]() { return c_.secrete(d, nullptr); }, &vs);
        if (rc == PCG_OK)
            rc = pick({128, 256, 512, 1024}, [&](int b) { m_.int_block = b; },
                      [&]() { return m_.integrate(c_, -1.0f, nullptr); }, &vi);
        ctx->launches = launches0;   // tuning launches are not the caller's work
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        PCG_CU(ctx, cudaMemcpyAsync(c_.soa.p, b_soa.p, c_.soa.bytes, cudaMemcpyDeviceToDevice, st));
        PCG_CU(ctx, cudaMemcpyAsync(c_.pos64.p, b_pos.p, c_.pos64.bytes, cudaMemcpyDeviceToDevice, st));
        PCG_CU(ctx, cudaMemcpyAsync(d.dens.p, b_dens.p, d.dens.bytes, cudaMemcpyDeviceToDevice, st));
        PCG_CU(ctx, cudaStreamSynchronize(st));
        if (rc != PCG_OK) return rc;
        c_.order_dirty = order_dirty;   // the SoA is back as it was: so is the secretion order
        T.store(kf, vf);
        T.store(ks, vs);
        T.store(kb, vb);
        T.store(ki, vi);
    }
    if (!pin_f) {
        m_.fshape.block = vf / 1000;
        m_.fshape.queue = vf % 1000;
    }
    if (!pin_t) {
        c_.sec_block = vs;
        m_.bin_block = vb;
        m_.int_block = vi;
    }
    return PCG_OK;
}

uint64_t Batch::count_launches(bool mech) const
{
    uint64_t k = d.launches_per_step();
    if (c_.n) k += 1;
    if (mech && c_.n) {
        k += m_.launches_forces(c_.n) - 1 + 1;   // bin..forces (memset excluded) + integrate
        // the secretion order after the voxel refresh: sort passes, run list, constants
        if (any_refresh) k += c_.order_launches();
    }
    return k;
}

// One main-loop sub-step; 'timed' records phase events.
int Batch::run_step(bool mech, bool timed, const uint8_t* mask)
{
    cudaStream_t st = ctx->stream;
    if (timed) PCG_CU(ctx, cudaEventRecord(ev[0], st));
    for (int a = 0; a < 3; ++a) {
        PCG_TRY(d.sweep(a, true, mask));
        if (timed) PCG_CU(ctx, cudaEventRecord(ev[1 + a], st));
    }
    if (c_.n) PCG_TRY(c_.secrete(d, mask));
    if (timed) PCG_CU(ctx, cudaEventRecord(ev[4], st));
    if (mech && c_.n) {
        PCG_TRY(m_.binsort(c_, mask));
        if (timed) PCG_CU(ctx, cudaEventRecord(ev[5], st));
        PCG_TRY(m_.force_pass(c_, mask));
        if (timed) PCG_CU(ctx, cudaEventRecord(ev[6], st));
        PCG_TRY(m_.integrate(c_, -1.0f, mask));
        if (any_refresh) PCG_TRY(c_.build_order(d.total_vox));
        if (timed) PCG_CU(ctx, cudaEventRecord(ev[7], st));
    }
    return PCG_OK;
}

int Batch::capture(bool mech, cudaGraphExec_t* out, uint64_t* launches, int n_diff)
{
    cudaStream_t st = ctx->stream;
    const uint64_t before = ctx->launches;
    PCG_CU(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const uint8_t* mask = masked ? mask_d.as<uint8_t>() : nullptr;
    int rc = PCG_OK;
    for (int k = 0; k < n_diff && rc == PCG_OK; ++k) rc = run_step(false, false, mask);   // sub-steps before mech
    if (rc == PCG_OK) rc = run_step(mech, false, mask);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != PCG_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "end capture");
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "graph instantiate");
    *launches = ctx->launches - before;
    ctx->launches = before;   // captured, not executed
    c_.order_dirty = false;   // ordering is rebuilt inside the mechanics graph when needed
    return PCG_OK;
}

int Batch::step(int n_steps)
{
    if (n_steps < 0) return fail(ctx, PCG_ERR_INVALID, "n_steps < 0");
    cudaStream_t st = ctx->stream;
    for (int s = 0; s < n_steps; ++s) {
        if (!profile && g_period && accum == 0.0 && n_steps - s >= period_len) {
            // a whole period: the accumulator fires on its last sub-step and resets
            PCG_CU(ctx, cudaGraphLaunch(g_period, st));
            ctx->launches += launches_period;
            s += period_len - 1;
            diff_steps += static_cast<uint64_t>(period_len);
            mech_steps++;
            m_.sorder_valid = false;
            continue;
        }
        accum += dt_diff;
        const bool mech = accum >= dt_mech - 0.5 * dt_diff;
        if (mech) accum = 0.0;
        if (profile) {
            PCG_TRY(run_step(mech, true, nullptr));
            PCG_CU(ctx, cudaEventSynchronize(mech ? ev[7] : ev[4]));
            float ms = 0;
            for (int a = 0; a < 3; ++a) {
                PCG_CU(ctx, cudaEventElapsedTime(&ms, ev[a], ev[a + 1]));
                phase_ms[a] += ms;
            }
            PCG_CU(ctx, cudaEventElapsedTime(&ms, ev[3], ev[4]));
            phase_ms[3] += ms;
            if (mech && c_.n) {
                PCG_CU(ctx, cudaEventElapsedTime(&ms, ev[4], ev[5]));
                phase_ms[4] += ms;
                PCG_CU(ctx, cudaEventElapsedTime(&ms, ev[5], ev[6]));
                phase_ms[5] += ms;
                PCG_CU(ctx, cudaEventElapsedTime(&ms, ev[6], ev[7]));
                phase_ms[6] += ms;
            }
            sweep_steps++;
        } else if (use_graphs) {
            PCG_CU(ctx, cudaGraphLaunch(mech ? g_mech : g_diff, st));
            ctx->launches += mech ? launches_mech : launches_diff;
        } else {
            PCG_TRY(run_step(mech, false, nullptr));
        }
        if (mech) {
            mech_steps++;
            m_.sorder_valid = false;   // binned again, stable order not made
        }
        diff_steps++;
    }
    return PCG_OK;
}

int Batch::step_masked(const uint8_t* mask_host, bool any_mech)
{
    if (!masked) return fail(ctx, PCG_ERR_INVALID, "batch was not created for masked steps");
    cudaStream_t st = ctx->stream;
    PCG_CU(ctx, cudaMemcpyAsync(mask_d.p, mask_host, mask_d.bytes, cudaMemcpyHostToDevice, st));
    if (use_graphs) {
        PCG_CU(ctx, cudaGraphLaunch(any_mech ? g_mech : g_diff, st));
        ctx->launches += any_mech ? launches_mech : launches_diff;
    } else {
        PCG_TRY(run_step(any_mech, false, mask_d.as<uint8_t>()));
    }
    diff_steps++;
    if (any_mech) {
        mech_steps++;
        m_.sorder_valid = false;
    }
    return PCG_OK;
}

int Batch::set_diagnostics(bool on)
{
    if (m_.diag == on) return PCG_OK;
    m_.diag = on;
    if (!use_graphs) return PCG_OK;
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    if (g_mech) {
        cudaGraphExecDestroy(g_mech);
        g_mech = nullptr;
    }
    PCG_TRY(capture(true, &g_mech, &launches_mech));
    if (!g_period) return PCG_OK;
    cudaGraphExecDestroy(g_period);
    g_period = nullptr;
    return capture(true, &g_period, &launches_period, period_len - 1);
}

std::string Batch::describe() const
{
    std::ostringstream o;
    o << d.describe() << "forces(block=" << m_.fshape.block << ",queue=" << m_.fshape.queue
      << ") secrete(block=" << c_.sec_block << ") bin(block=" << m_.bin_block << ") integrate(block="
      << m_.int_block << ") graphs=" << (use_graphs ? 1 : 0)
      << " launches/step=" << launches_diff << "/" << launches_mech;
    return o.str();
}

}  // namespace pcg

struct pcg_batch {
    Batch b;
    std::string desc;
};

extern "C" {

uint64_t pcg_instance_bytes(const pcg_instance_desc* inst) { return inst ? instance_bytes(*inst) : 0; }

pcg_status pcg_batch_create(pcg_ctx* ctx, const pcg_instance_desc* inst, uint32_t n, const pcg_batch_options* opt,
                            pcg_batch** out)
{
    if (!ctx || !out || (!inst && n)) return PCG_ERR_INVALID;
    *out = nullptr;
    pcg_batch* b = new (std::nothrow) pcg_batch();
    if (!b) return PCG_ERR_OOM;
    int rc = b->b.create(ctx, inst, n, opt);
    if (rc != PCG_OK) {
        delete b;
        return rc;
    }
    ctx_retain(ctx);
    *out = b;
    return PCG_OK;
}

pcg_status pcg_batch_destroy(pcg_batch* b)
{
    if (!b) return PCG_OK;
    pcg_ctx* ctx = b->b.ctx;
    cudaStreamSynchronize(ctx->stream);
    delete b;
    ctx_release(ctx);
    return PCG_OK;
}

pcg_status pcg_batch_step(pcg_batch* b, int n) { return b ? b->b.step(n) : PCG_ERR_INVALID; }

pcg_status pcg_batch_download_density(pcg_batch* b, uint32_t i, float* host, size_t n)
{
    if (!b || !host || i >= b->b.d.inst.size()) return PCG_ERR_INVALID;
    const DiffInstance& di = b->b.d.inst[i];
    if (n != di.nvox() * di.g.n_substrates) return fail(b->b.ctx, PCG_ERR_INVALID, "density size mismatch");
    return b->b.d.download(i, host);
}

pcg_status pcg_batch_download_cells(pcg_batch* b, uint32_t i, float* soa, uint32_t soa_max)
{
    if (!b || !soa || i >= b->b.ncell.size()) return PCG_ERR_INVALID;
    const CellInst& ci = b->b.c_.h_inst[i];
    if (soa_max < ci.n_cells) return fail(b->b.ctx, PCG_ERR_INVALID, "soa_max_cells < n_cells");
    PCG_TRY(b->b.c_.download_soa(ci.cell_off, ci.n_cells, soa, soa_max, 0, NUM_FIELDS));
    PCG_CU(b->b.ctx, cudaStreamSynchronize(b->b.ctx->stream));
    return PCG_OK;
}

pcg_status pcg_batch_download_positions64(pcg_batch* b, uint32_t i, double* xyz, uint32_t n_cells)
{
    if (!b || i >= b->b.ncell.size() || (!xyz && n_cells)) return PCG_ERR_INVALID;
    const CellInst& ci = b->b.c_.h_inst[i];
    if (n_cells != ci.n_cells) return fail(b->b.ctx, PCG_ERR_INVALID, "n_cells must equal the instance's cell count");
    return b->b.c_.download_positions(ci.cell_off, n_cells, xyz);
}

pcg_status pcg_batch_upload_cells(pcg_batch* b, uint32_t i, const float* soa, uint32_t soa_max)
{
    if (!b || !soa || i >= b->b.ncell.size()) return PCG_ERR_INVALID;
    const CellInst& ci = b->b.c_.h_inst[i];
    if (soa_max < ci.n_cells) return fail(b->b.ctx, PCG_ERR_INVALID, "soa_max_cells < n_cells");
    PCG_TRY(b->b.c_.upload_soa(ci.cell_off, ci.n_cells, soa, soa_max, 0, NUM_FIELDS));
    PCG_CU(b->b.ctx, cudaStreamSynchronize(b->b.ctx->stream));
    // volumes and voxel indices may have changed: rebuild the secretion constants and order now
    PCG_TRY(b->b.c_.prepare_secretion(b->b.dt_diff, b->b.d.total_vox));
    return PCG_OK;
}

namespace {

int ensure_copy_streams(pcg_ctx* ctx)
{
    if (ctx->h2d) return PCG_OK;
    PCG_CU(ctx, cudaStreamCreateWithFlags(&ctx->h2d, cudaStreamNonBlocking));
    PCG_CU(ctx, cudaStreamCreateWithFlags(&ctx->d2h, cudaStreamNonBlocking));
    for (auto& e : ctx->copy_ev) PCG_CU(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return PCG_OK;
}

// An event recorded once on the context stream when made, so that the first
// wait on it passes.
int ensure_event(pcg_ctx* ctx, cudaEvent_t* e)
{
    if (*e) return PCG_OK;
    PCG_CU(ctx, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    PCG_CU(ctx, cudaEventRecord(*e, ctx->stream));
    return PCG_OK;
}

int ensure_stage(pcg_ctx* ctx, DevBuf& b, size_t bytes)
{
    if (b.bytes >= bytes) return PCG_OK;
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->h2d) PCG_CU(ctx, cudaStreamSynchronize(ctx->h2d));
    if (ctx->d2h) PCG_CU(ctx, cudaStreamSynchronize(ctx->d2h));
    b.release();
    PCG_CU(ctx, b.alloc(bytes));
    return PCG_OK;
}

// device -> staging on the context stream, then staging -> host on the
// copy stream; 'done' gates the next reuse of the staging buffer
int staged_download(pcg_ctx* ctx, DevBuf& stage, cudaEvent_t* ready, cudaEvent_t* done, void* host,
                    const void* src, size_t spitch, size_t width, size_t rows)
{
    PCG_TRY(ensure_copy_streams(ctx));
    PCG_TRY(ensure_stage(ctx, stage, width * rows));
    PCG_TRY(ensure_event(ctx, ready));
    PCG_TRY(ensure_event(ctx, done));
    PCG_CU(ctx, cudaStreamWaitEvent(ctx->stream, *done, 0));
    PCG_CU(ctx, cudaMemcpy2DAsync(stage.p, width, src, spitch, width, rows, cudaMemcpyDeviceToDevice, ctx->stream));
    PCG_CU(ctx, cudaEventRecord(*ready, ctx->stream));
    PCG_CU(ctx, cudaStreamWaitEvent(ctx->d2h, *ready, 0));
    PCG_CU(ctx, cudaMemcpyAsync(host, stage.p, width * rows, cudaMemcpyDeviceToHost, ctx->d2h));
    PCG_CU(ctx, cudaEventRecord(*done, ctx->d2h));
    return PCG_OK;
}

}  // namespace

pcg_status pcg_batch_upload_all_cells(pcg_batch* b, const float* soa, uint64_t n_floats)
{
    if (!b || !soa) return PCG_ERR_INVALID;
    Batch& B = b->b;
    Cells& c = B.c_;
    pcg_ctx* ctx = B.ctx;
    if (n_floats != static_cast<uint64_t>(NUM_FIELDS) * c.n) return fail(ctx, PCG_ERR_INVALID, "size mismatch");
    if (c.n == 0) return PCG_OK;
    // host -> staging on the copy stream (once the previous upload has left
    // the staging buffer), then staging -> the cell SoA on the context stream
    const size_t row = static_cast<size_t>(c.n) * sizeof(float);
    PCG_TRY(ensure_copy_streams(ctx));
    PCG_TRY(ensure_stage(ctx, B.stage_in, row * NUM_FIELDS));
    PCG_TRY(ensure_event(ctx, &B.ev_in_done));
    PCG_TRY(ensure_event(ctx, &B.ev_in_used));
    PCG_CU(ctx, cudaStreamWaitEvent(ctx->h2d, B.ev_in_used, 0));
    PCG_CU(ctx, cudaMemcpyAsync(B.stage_in.p, soa, row * NUM_FIELDS, cudaMemcpyHostToDevice, ctx->h2d));
    PCG_CU(ctx, cudaEventRecord(B.ev_in_done, ctx->h2d));
    PCG_CU(ctx, cudaStreamWaitEvent(ctx->stream, B.ev_in_done, 0));
    PCG_CU(ctx, cudaMemcpy2DAsync(c.soa.p, static_cast<size_t>(c.max_cells) * sizeof(float), B.stage_in.p, row, row,
                                  NUM_FIELDS, cudaMemcpyDeviceToDevice, ctx->stream));
    PCG_CU(ctx, cudaEventRecord(B.ev_in_used, ctx->stream));
    c.coef_dirty = c.order_dirty = true;   // volumes and voxel indices came with the fields
    PCG_TRY(c.prepare_secretion(B.dt_diff, B.d.total_vox));
    return PCG_OK;
}

pcg_status pcg_batch_download_all_cells(pcg_batch* b, float* soa, uint64_t n_floats)
{
    if (!b || !soa) return PCG_ERR_INVALID;
    Batch& B = b->b;
    Cells& c = B.c_;
    if (n_floats != static_cast<uint64_t>(NUM_FIELDS) * c.n) return fail(B.ctx, PCG_ERR_INVALID, "size mismatch");
    if (c.n == 0) return PCG_OK;
    return staged_download(B.ctx, B.stage_cells, &B.ev_cells_ready, &B.ev_cells_done, soa, c.soa.p,
                           static_cast<size_t>(c.max_cells) * sizeof(float), static_cast<size_t>(c.n) * sizeof(float),
                           NUM_FIELDS);
}

pcg_status pcg_batch_download_cell_fields(pcg_batch* b, float* soa, uint64_t n_floats, uint32_t field_mask)
{
    if (!b || !soa) return PCG_ERR_INVALID;
    Batch& B = b->b;
    Cells& c = B.c_;
    pcg_ctx* ctx = B.ctx;
    if (n_floats != static_cast<uint64_t>(NUM_FIELDS) * c.n) return fail(ctx, PCG_ERR_INVALID, "size mismatch");
    if (field_mask >> NUM_FIELDS) return fail(ctx, PCG_ERR_INVALID, "field mask names a field past the 28");
    if (c.n == 0 || field_mask == 0) return PCG_OK;
    // runs of consecutive fields: device -> staging (packed) on the context
    // stream, staging -> each run's place in the host SoA on the copy stream
    std::vector<std::pair<uint32_t, uint32_t>> runs;
    for (uint32_t f = 0; f < static_cast<uint32_t>(NUM_FIELDS);) {
        if (!(field_mask >> f & 1u)) {
            ++f;
            continue;
        }
        uint32_t e = f;
        while (e < static_cast<uint32_t>(NUM_FIELDS) && (field_mask >> e & 1u)) ++e;
        runs.emplace_back(f, e);
        f = e;
    }
    const size_t row = static_cast<size_t>(c.n) * sizeof(float);
    const size_t nsel = static_cast<size_t>(__builtin_popcount(field_mask));
    PCG_TRY(ensure_copy_streams(ctx));
    PCG_TRY(ensure_stage(ctx, B.stage_cells, row * nsel));
    PCG_TRY(ensure_event(ctx, &B.ev_cells_ready));
    PCG_TRY(ensure_event(ctx, &B.ev_cells_done));
    PCG_CU(ctx, cudaStreamWaitEvent(ctx->stream, B.ev_cells_done, 0));
    size_t at = 0;
    for (const auto& r : runs) {
        PCG_CU(ctx, cudaMemcpy2DAsync(static_cast<char*>(B.stage_cells.p) + at * row, row,
                                      c.soa.as<float>() + static_cast<size_t>(r.first) * c.max_cells,
                                      static_cast<size_t>(c.max_cells) * sizeof(float), row, r.second - r.first,
                                      cudaMemcpyDeviceToDevice, ctx->stream));
        at += r.second - r.first;
    }
    PCG_CU(ctx, cudaEventRecord(B.ev_cells_ready, ctx->stream));
    PCG_CU(ctx, cudaStreamWaitEvent(ctx->d2h, B.ev_cells_ready, 0));
    at = 0;
    for (const auto& r : runs) {
        PCG_CU(ctx, cudaMemcpyAsync(soa + static_cast<size_t>(r.first) * c.n,
                                    static_cast<char*>(B.stage_cells.p) + at * row, (r.second - r.first) * row,
                                    cudaMemcpyDeviceToHost, ctx->d2h));
        at += r.second - r.first;
    }
    PCG_CU(ctx, cudaEventRecord(B.ev_cells_done, ctx->d2h));
    return PCG_OK;
}

pcg_status pcg_batch_upload_cell_fields(pcg_batch* b, const float* soa, uint64_t n_floats, uint32_t field_mask)
{
    if (!b || !soa) return PCG_ERR_INVALID;
    Batch& B = b->b;
    Cells& c = B.c_;
    pcg_ctx* ctx = B.ctx;
    if (n_floats != static_cast<uint64_t>(NUM_FIELDS) * c.n) return fail(ctx, PCG_ERR_INVALID, "size mismatch");
    if (field_mask >> NUM_FIELDS) return fail(ctx, PCG_ERR_INVALID, "field mask names a field past the 28");
    if (c.n == 0 || field_mask == 0) return PCG_OK;
    // runs of consecutive fields: each run's place in the host SoA -> staging
    // (packed) on the copy stream, staging -> the SoA on the context stream
    std::vector<std::pair<uint32_t, uint32_t>> runs;
    for (uint32_t f = 0; f < static_cast<uint32_t>(NUM_FIELDS);) {
        if (!(field_mask >> f & 1u)) {
            ++f;
            continue;
        }
        uint32_t e = f;
        while (e < static_cast<uint32_t>(NUM_FIELDS) && (field_mask >> e & 1u)) ++e;
        runs.emplace_back(f, e);
        f = e;
    }
    const size_t row = static_cast<size_t>(c.n) * sizeof(float);
    const size_t nsel = static_cast<size_t>(__builtin_popcount(field_mask));
    PCG_TRY(ensure_copy_streams(ctx));
    PCG_TRY(ensure_stage(ctx, B.stage_in, row * nsel));
    PCG_TRY(ensure_event(ctx, &B.ev_in_done));
    PCG_TRY(ensure_event(ctx, &B.ev_in_used));
    PCG_CU(ctx, cudaStreamWaitEvent(ctx->h2d, B.ev_in_used, 0));
    size_t at = 0;
    for (const auto& r : runs) {
        PCG_CU(ctx, cudaMemcpyAsync(static_cast<char*>(B.stage_in.p) + at * row,
                                    soa + static_cast<size_t>(r.first) * c.n, (r.second - r.first) * row,
                                    cudaMemcpyHostToDevice, ctx->h2d));
        at += r.second - r.first;
    }
    PCG_CU(ctx, cudaEventRecord(B.ev_in_done, ctx->h2d));
    PCG_CU(ctx, cudaStreamWaitEvent(ctx->stream, B.ev_in_done, 0));
    at = 0;
    for (const auto& r : runs) {
        PCG_CU(ctx, cudaMemcpy2DAsync(c.soa.as<float>() + static_cast<size_t>(r.first) * c.max_cells,
                                      static_cast<size_t>(c.max_cells) * sizeof(float),
                                      static_cast<const char*>(B.stage_in.p) + at * row, row, row,
                                      r.second - r.first, cudaMemcpyDeviceToDevice, ctx->stream));
        at += r.second - r.first;
    }
    PCG_CU(ctx, cudaEventRecord(B.ev_in_used, ctx->stream));
    // volumes feed the secretion constants, voxel indices the secretion order
    if (field_mask >> F_TOTAL_VOL & 1u) c.coef_dirty = true;
    if (field_mask >> F_VOXEL_IDX & 1u) c.order_dirty = true;
    if (c.coef_dirty || c.order_dirty) PCG_TRY(c.prepare_secretion(B.dt_diff, B.d.total_vox));
    return PCG_OK;
}

pcg_status pcg_batch_download_all_density(pcg_batch* b, float* host, uint64_t n_floats)
{
    if (!b || !host) return PCG_ERR_INVALID;
    Batch& B = b->b;
    if (n_floats != B.d.dens_elems) return fail(B.ctx, PCG_ERR_INVALID, "size mismatch");
    if (n_floats == 0) return PCG_OK;
    const size_t bytes = n_floats * sizeof(float);
    return staged_download(B.ctx, B.stage_dens, &B.ev_dens_ready, &B.ev_dens_done, host, B.d.dens.p, bytes, bytes, 1);
}

pcg_status pcg_batch_density_layout(pcg_batch* b, uint32_t i, uint64_t* off, uint64_t* row_pitch, uint64_t* pitch,
                                    uint64_t* arena)
{
    if (!b || i >= b->b.d.inst.size()) return PCG_ERR_INVALID;
    if (off) *off = b->b.d.inst[i].dens_off;
    if (row_pitch) *row_pitch = b->b.d.inst[i].px;
    if (pitch) *pitch = b->b.d.inst[i].pitch;
    if (arena) *arena = b->b.d.dens_elems;
    return PCG_OK;
}

pcg_status pcg_batch_totals(pcg_batch* b, uint64_t* voxels, uint64_t* vs, uint64_t* cells)
{
    if (!b) return PCG_ERR_INVALID;
    if (voxels) *voxels = b->b.d.total_vox;
    if (vs) *vs = b->b.d.total_vox_sub;
    if (cells) *cells = b->b.c_.n;
    return PCG_OK;
}

pcg_status pcg_batch_sweep_units(pcg_batch* b, uint64_t* plane_units, uint64_t* all_units)
{
    if (!b) return PCG_ERR_INVALID;
    uint64_t pu = 0;
    for (const auto& pl : b->b.d.planes) pu += pl.units;
    for (const auto& pl : b->b.d.zplanes) pu += pl.units;
    if (plane_units) *plane_units = pu;
    if (all_units) *all_units = b->b.d.sweep_units_per_step();
    return PCG_OK;
}

pcg_status pcg_batch_step_launches(pcg_batch* b, uint64_t* ld, uint64_t* lm)
{
    if (!b) return PCG_ERR_INVALID;
    if (ld) *ld = b->b.launches_diff;
    if (lm) *lm = b->b.launches_mech;
    return PCG_OK;
}

pcg_status pcg_batch_phase_times(pcg_batch* b, float* ms, uint64_t* n_sweep_steps, int reset)
{
    if (!b) return PCG_ERR_INVALID;
    if (ms)
        for (int q = 0; q < PCG_N_PHASES; ++q) ms[q] = static_cast<float>(b->b.phase_ms[q]);
    if (n_sweep_steps) *n_sweep_steps = b->b.sweep_steps;
    if (reset) {
        for (int q = 0; q < PCG_N_PHASES; ++q) b->b.phase_ms[q] = 0.0;
        b->b.sweep_steps = 0;
    }
    return PCG_OK;
}

pcg_status pcg_batch_set_diagnostics(pcg_batch* b, int on)
{
    if (!b) return PCG_ERR_INVALID;
    return b->b.set_diagnostics(on != 0);
}

pcg_status pcg_batch_mech_bins(pcg_batch* b, uint32_t i, uint32_t* start, uint32_t* sorted_cells,
                               uint32_t* nbr_count, uint32_t* nbr_hash)
{
    if (!b || i >= b->b.ncell.size()) return PCG_ERR_INVALID;
    Batch& B = b->b;
    pcg_ctx* ctx = B.ctx;
    if ((nbr_count || nbr_hash) && !B.m_.diag) return fail(ctx, PCG_ERR_INVALID, "diagnostics are off");
    const CellInst& ci = B.c_.h_inst[i];
    const size_t V = static_cast<size_t>(ci.mnx) * ci.mny * ci.mnz;
    if (sorted_cells) PCG_TRY(B.m_.stable_order(B.c_.n));   // from the last binning, if not yet made
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    std::vector<uint32_t> st(V + 1);
    PCG_CU(ctx, cudaMemcpy(st.data(), B.m_.start.as<uint32_t>() + ci.mvox_base, (V + 1) * sizeof(uint32_t),
                           cudaMemcpyDeviceToHost));
    const uint32_t first = st[0];
    if (st[V] - first != ci.n_cells) return fail(ctx, PCG_ERR_INVALID, "no mechanics step has binned this instance");
    if (start)
        for (size_t v = 0; v <= V; ++v) start[v] = st[v] - first;
    if (sorted_cells && ci.n_cells) {
        PCG_CU(ctx, cudaMemcpy(sorted_cells, B.m_.sorder.as<uint32_t>() + first, ci.n_cells * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost));
        for (uint32_t q = 0; q < ci.n_cells; ++q) sorted_cells[q] -= ci.cell_off;
    }
    if (nbr_count && ci.n_cells)
        PCG_CU(ctx, cudaMemcpy(nbr_count, B.m_.dcnt.as<uint32_t>() + ci.cell_off, ci.n_cells * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost));
    if (nbr_hash && ci.n_cells)
        PCG_CU(ctx, cudaMemcpy(nbr_hash, B.m_.dhash.as<uint32_t>() + ci.cell_off, ci.n_cells * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost));
    return PCG_OK;
}

pcg_status pcg_batch_set_profile(pcg_batch* b, int on)
{
    if (!b) return PCG_ERR_INVALID;
    b->b.profile = on != 0;
    return PCG_OK;
}

const char* pcg_batch_describe(pcg_batch* b)
{
    if (!b) return "";
    b->desc = b->b.describe();
    return b->desc.c_str();
}

}  // extern "C"
