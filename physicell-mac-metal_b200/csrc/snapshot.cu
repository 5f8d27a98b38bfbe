// snapshot.cu — writeMatlabSnapshots (src/output_writer.cpp:295-452,
// src/matlab_writer.cpp:5-49) as an asynchronous device -> host snapshot.
//
// Each matrix is assembled on the device in the file's own layout (MATLAB v4,
// one full double matrix, column-major: one column per voxel or per cell) by
// a kernel on the snapshot's stream, which starts after the work already
// queued on the context stream; the context stream waits only for that
// kernel, so the simulation goes on while the matrix is copied to pinned
// memory and a host callback writes the file.  Values are formed with the
// reference's own arithmetic (FP32 voxel centres and surface areas widened
// to double), so the files are byte-identical to the reference writer's.
//
// Cell columns come from what the device holds: the 28-field SoA and the
// secretion rates.  The reference fills the columns of its CPU-side
// phenotype arrays (cycle, death, volume rates, interactions, ...) with
// fixed defaults when those arrays are absent; the snapshot writes the same
// defaults.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <string>

#include "capi.h"

namespace pcg {

namespace {

// Rows of a cell column (output_writer.cpp:311-438) for S substrates and
// T cell types.
__host__ __device__ constexpr uint32_t cell_rows(uint32_t S, uint32_t T) { return 71u + 7u * T + 8u * S; }

__global__ void k_mat_microenvironment(const float* __restrict__ dens, uint64_t sub_pitch, uint32_t px,
                                       pcg_grid_params g, double* __restrict__ out)
{
    const uint64_t nv = static_cast<uint64_t>(g.nx) * g.ny * g.nz;
    const uint32_t rows = 4u + g.n_substrates;
    const float vvol = __fmul_rn(__fmul_rn(g.dx, g.dy), g.dz);
    for (uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; v < nv;
         v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t iz = static_cast<uint32_t>(v / (static_cast<uint64_t>(g.nx) * g.ny));
        const uint32_t rem = static_cast<uint32_t>(v % (static_cast<uint64_t>(g.nx) * g.ny));
        const uint32_t iy = rem / g.nx, ix = rem % g.nx;
        double* c = out + v * rows;
        c[0] = __fadd_rn(g.x_min, __fmul_rn(__fadd_rn(static_cast<float>(ix), 0.5f), g.dx));
        c[1] = __fadd_rn(g.y_min, __fmul_rn(__fadd_rn(static_cast<float>(iy), 0.5f), g.dy));
        c[2] = __fadd_rn(g.z_min, __fmul_rn(__fadd_rn(static_cast<float>(iz), 0.5f), g.dz));
        c[3] = vvol;
        const uint64_t row = static_cast<uint64_t>(iz) * g.ny + iy;
        for (uint32_t s = 0; s < g.n_substrates; ++s) c[4 + s] = dens[s * sub_pitch + row * px + ix];
    }
}

// One column per cell, in the reference's order.
__global__ void k_mat_cells(const float* __restrict__ soa, uint32_t stride, uint32_t n, const double* __restrict__ rates,
                            uint64_t rate_cap, uint32_t S, uint32_t T, double* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    auto f = [&](int fld) { return soa[static_cast<size_t>(fld) * stride + i]; };
    auto u = [&](int fld) { return __float_as_uint(soa[static_cast<size_t>(fld) * stride + i]); };
    double* c = out + static_cast<size_t>(i) * cell_rows(S, T);
    uint32_t r = 0;
    auto put = [&](double x) { c[r++] = x; };
    // compatibility entries
    put(static_cast<double>(i));
    put(f(F_POS_X));
    put(f(F_POS_Y));
    put(f(F_POS_Z));
    put(f(F_TOTAL_VOL));
    put(static_cast<double>(u(23)));      // cell_type
    put(5.0);                             // cycle_model_code (CPU-side)
    put(static_cast<double>(u(24)));      // current_phase
    put(0.0);                             // elapsed_time_in_phase (CPU-side)
    put(f(12));                           // nuclear_volume
    put(__fsub_rn(f(F_TOTAL_VOL), f(12)));
    put(0.75);                            // fluid_fraction (CPU-side)
    put(0.0);                             // calcified_fraction (CPU-side)
    put(0.0); put(0.0); put(0.0);         // orientation
    put(0.0);                             // polarity
    // state
    put(f(F_VEL_X));
    put(f(F_VEL_Y));
    put(f(F_VEL_Z));
    put(f(F_PRESSURE));
    put(1.0); put(0.0); put(0.0);         // nuclei, attack time, contact_BM
    // cycle and death
    put(0.0);                             // transition_rate_01 (CPU-side)
    put(0.0);                             // elapsed_time_in_phase (CPU-side)
    put(u(F_IS_ALIVE) ? 0.0 : 1.0);
    put(0.0);                             // current_death_model (CPU-side)
    put(0.0);                             // apoptosis rate
    put(0.0);                             // necrosis_rate (CPU-side)
    // volume (CPU-side rates and targets)
    for (int k = 0; k < 7; ++k) put(0.0);
    // geometry
    const float rad = f(F_RADIUS);
    put(rad);
    put(f(10));                           // nuclear_radius
    put(__fmul_rn(__fmul_rn(4.0f * 3.14159f, rad), rad));
    // mechanics
    put(f(F_ADHESION));
    put(0.0);
    put(f(F_REPULSION));
    put(0.0);
    for (uint32_t t = 0; t < T; ++t) put(1.0);   // adhesion affinities
    put(f(F_REL_MAX_ADH));
    put(12.0);                            // max_attachments
    put(0.0); put(0.0); put(0.0);         // attachment constants (CPU-side)
    // motility
    const float sp = f(F_MOT_SPEED);
    put(sp > 0.0f ? 1.0 : 0.0);
    put(15.0);                            // persistence_time
    put(sp);
    put(f(18)); put(f(19)); put(f(20));   // motility direction
    put(f(17));                           // motility_bias
    put(0.0); put(0.0); put(0.0);         // motility_vector
    put(0.0);                             // chemotaxis_index
    put(1.0);                             // chemotaxis_dir
    for (uint32_t s = 0; s < S; ++s) put(0.0);   // chemotactic sensitivities
    // secretion: rates arrays [q * cap + cell * S + s]
    for (int q = 0; q < 4; ++q)
        for (uint32_t s = 0; s < S; ++s) put(rates[static_cast<uint64_t>(q) * rate_cap + static_cast<uint64_t>(i) * S + s]);
    // molecular
    for (uint32_t s = 0; s < 3u * S; ++s) put(0.0);
    // interactions
    put(0.0); put(0.0); put(0.0);         // phagocytosis rates (CPU-side)
    for (uint32_t t = 0; t < T; ++t) put(0.0);   // live phagocytosis
    for (uint32_t t = 0; t < T; ++t) put(0.0);   // attack rates
    for (uint32_t t = 0; t < T; ++t) put(1.0);   // immunogenicities
    put(0.0); put(0.0); put(0.0); put(0.0);      // attacking cell, damage rate, duration, reserved
    for (uint32_t t = 0; t < 3u * T; ++t) put(0.0);   // fusion, transformation, reserved
    // integrity
    put(0.0); put(0.0); put(0.0);
}

struct Job {
    std::string path, name;
    uint32_t rows = 0, cols = 0;
    DevBuf dev;
    HostBuf host;
    std::atomic<int> done{0};
    std::atomic<int> ok{1};
};

// Host callback on the snapshot stream: no CUDA calls, file I/O only.
void CUDART_CB write_job(void* p)
{
    Job* j = static_cast<Job*>(p);
    FILE* fp = std::fopen(j->path.c_str(), "wb");
    bool ok = fp != nullptr;
    if (ok) {
        const uint32_t head[5] = {0u, j->rows, j->cols, 0u, static_cast<uint32_t>(j->name.size() + 1)};
        ok = std::fwrite(head, sizeof head, 1, fp) == 1;
        ok = ok && std::fwrite(j->name.c_str(), 1, j->name.size() + 1, fp) == j->name.size() + 1;
        const size_t n = static_cast<size_t>(j->rows) * j->cols;
        ok = ok && std::fwrite(j->host.p, sizeof(double), n, fp) == n;
        ok = (std::fclose(fp) == 0) && ok;
    }
    j->ok.store(ok ? 1 : 0);
    j->done.store(1);
}

}  // namespace

}  // namespace pcg

using namespace pcg;

struct pcg_snapshot {
    pcg_ctx* ctx = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t queued = nullptr, built = nullptr;
    std::deque<std::unique_ptr<Job>> jobs;
    bool failed = false;
    std::string failed_path;

    // release the buffers of finished jobs and remember failures
    void reap(bool all_done)
    {
        while (!jobs.empty() && (all_done || jobs.front()->done.load())) {
            if (!jobs.front()->ok.load()) {
                failed = true;
                failed_path = jobs.front()->path;
            }
            jobs.pop_front();
        }
    }
};

namespace {

// Order the snapshot stream after the context's queued work, build the
// matrix with 'launch', let the context stream wait for the build only, then
// copy and write asynchronously.
template <class L>
int submit(pcg_snapshot* s, const std::string& path, const char* name, uint32_t rows, uint32_t cols, L launch)
{
    pcg_ctx* ctx = s->ctx;
    s->reap(false);
    std::unique_ptr<Job> j(new (std::nothrow) Job());
    if (!j) return PCG_ERR_OOM;
    j->path = path;
    j->name = name;
    j->rows = rows;
    j->cols = cols;
    const size_t bytes = static_cast<size_t>(rows) * cols * sizeof(double);
    {
        AllocStream pool_scope(s->st);
        PCG_CU(ctx, j->dev.alloc(bytes));
    }
    PCG_CU(ctx, j->host.alloc(bytes));
    PCG_CU(ctx, cudaEventRecord(s->queued, ctx->stream));
    PCG_CU(ctx, cudaStreamWaitEvent(s->st, s->queued, 0));
    PCG_CU(ctx, launch(j->dev.as<double>()));
    ctx->launches++;
    PCG_CU(ctx, cudaEventRecord(s->built, s->st));
    PCG_CU(ctx, cudaStreamWaitEvent(ctx->stream, s->built, 0));   // later work may change the source
    PCG_CU(ctx, cudaMemcpyAsync(j->host.p, j->dev.p, bytes, cudaMemcpyDeviceToHost, s->st));
    PCG_CU(ctx, cudaLaunchHostFunc(s->st, write_job, j.get()));
    s->jobs.push_back(std::move(j));
    return PCG_OK;
}

int snap_env(pcg_snapshot* s, const pcg_me* me, const std::string& path)
{
    const DiffInstance& di = me->d.inst[0];
    const pcg_grid_params g = di.g;
    const uint64_t nv = di.nvox();
    if (nv == 0) return PCG_OK;
    if (nv > 0xFFFFFFFFull) return fail(s->ctx, PCG_ERR_INVALID, "grid too large for a v4 matrix");
    const float* dens = me->d.dens.as<float>() + di.dens_off;
    return submit(s, path, "multiscale_microenvironment", 4u + g.n_substrates, static_cast<uint32_t>(nv),
                  [&](double* out) {
                      const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((nv + 255) / 256, 148 * 16));
                      k_mat_microenvironment<<<blocks, 256, 0, s->st>>>(dens, di.pitch, di.px, g, out);
                      return cudaGetLastError();
                  });
}

int snap_cells(pcg_snapshot* s, const pcg_cells* cells, uint32_t n_types, const std::string& path)
{
    const Cells& c = cells->c;
    if (c.n == 0) return PCG_OK;
    const uint32_t S = cells->S, T = std::max<uint32_t>(n_types, 1);
    const uint64_t cap = c.rates.bytes / (4 * sizeof(double));
    return submit(s, path, "cells", cell_rows(S, T), c.n, [&](double* out) {
        k_mat_cells<<<(c.n + 127) / 128, 128, 0, s->st>>>(c.soa.as<float>(), c.max_cells, c.n, c.rates.as<double>(),
                                                          cap, S, T, out);
        return cudaGetLastError();
    });
}

}  // namespace

extern "C" {

pcg_status pcg_snapshot_create(pcg_ctx* ctx, pcg_snapshot** out)
{
    if (!ctx || !out) return PCG_ERR_INVALID;
    *out = nullptr;
    pcg_snapshot* s = new (std::nothrow) pcg_snapshot();
    if (!s) return PCG_ERR_OOM;
    s->ctx = ctx;
    cudaError_t e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->queued, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->built, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (s->queued) cudaEventDestroy(s->queued);
        if (s->st) cudaStreamDestroy(s->st);
        delete s;
        return cuda_fail(ctx, e, "snapshot stream");
    }
    ctx_retain(ctx);
    *out = s;
    return PCG_OK;
}

pcg_status pcg_snapshot_wait(pcg_snapshot* s)
{
    if (!s) return PCG_ERR_INVALID;
    PCG_CU(s->ctx, cudaStreamSynchronize(s->st));
    s->reap(true);
    if (s->failed) {
        s->failed = false;
        return fail(s->ctx, PCG_ERR_INVALID, "could not write " + s->failed_path);
    }
    return PCG_OK;
}

pcg_status pcg_snapshot_destroy(pcg_snapshot* s)
{
    if (!s) return PCG_ERR_INVALID;
    const int rc = pcg_snapshot_wait(s);
    s->jobs.clear();
    cudaEventDestroy(s->queued);
    cudaEventDestroy(s->built);
    cudaStreamDestroy(s->st);
    pcg_ctx* ctx = s->ctx;
    delete s;
    ctx_release(ctx);
    return rc;
}

pcg_status pcg_snapshot_microenvironment(pcg_snapshot* s, const pcg_me* me, const char* path)
{
    if (!s || !me || !path) return PCG_ERR_INVALID;
    if (me->ctx != s->ctx) return fail(s->ctx, PCG_ERR_INVALID, "objects of different contexts");
    return snap_env(s, me, path);
}

pcg_status pcg_snapshot_cells(pcg_snapshot* s, const pcg_cells* cells, uint32_t n_cell_types, const char* path)
{
    if (!s || !cells || !path) return PCG_ERR_INVALID;
    if (cells->ctx != s->ctx) return fail(s->ctx, PCG_ERR_INVALID, "objects of different contexts");
    return snap_cells(s, cells, n_cell_types, path);
}

pcg_status pcg_snapshot_frame(pcg_snapshot* s, const pcg_me* me, const pcg_cells* cells, uint32_t n_cell_types,
                              const char* folder, int frame)
{
    if (!s || !folder) return PCG_ERR_INVALID;
    char name[64];
    if (cells) {
        std::snprintf(name, sizeof name, "/output%08d_cells.mat", frame);
        PCG_TRY(pcg_snapshot_cells(s, cells, n_cell_types, (std::string(folder) + name).c_str()));
    }
    if (me) {
        std::snprintf(name, sizeof name, "/output%08d_microenvironment0.mat", frame);
        PCG_TRY(pcg_snapshot_microenvironment(s, me, (std::string(folder) + name).c_str()));
    }
    return PCG_OK;
}

}  // extern "C"
