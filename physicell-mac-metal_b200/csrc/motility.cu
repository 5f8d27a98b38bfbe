// motility.cu — updateMotility (src/motility.cpp:179-293) on the device:
// one thread per cell, the persistent random walk with chemotaxis bias added
// to the velocity the force pass wrote.  FP64 throughout, round-to-nearest
// operations without contraction, so every value matches the CPU
// restatement except where the double sine / cosine of the random angles
// differ in their last place.  Draws come from a counter-based generator of
// (seed, cell, step, k): three rounds of the SplitMix64 finaliser (Steele,
// Lea and Flood, 2014) keep a run reproducible where the reference's
// std::random_device-seeded generator does not.
#include "capi.h"

namespace pcg {

namespace {

struct MotState {
    double* persistence;
    double* elapsed;
    const double* bias;
    double* vec;            // x, y, z arrays of n
    const uint32_t* is_motile;
    const uint32_t* restrict_2d;
    const int32_t* chem_index;
    const int32_t* chem_dir;
    const double* sens;     // n * n_sens, cell-major; null: single-substrate rule
    uint32_t n_sens;
    uint32_t n;
};

// The density of one instance in the library's pitched layout.
struct DensView {
    const float* base;      // substrate 0, voxel 0
    uint64_t sub_pitch;     // floats between substrates
    uint32_t px;            // floats between rows
    uint32_t nx, ny, nz, S;
    float dx, dy, dz, x_min, y_min, z_min;
};

constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double uniform(uint64_t seed, uint64_t cell, uint64_t step, uint32_t k)
{
    uint64_t h = mix64(seed ^ 0x9e3779b97f4a7c15ull);
    h = mix64(h ^ cell);
    h = mix64(h ^ step);
    h = mix64(h ^ static_cast<uint64_t>(k));
    return static_cast<double>(h >> 11) * 0x1.0p-53;
}

__device__ __forceinline__ int clampi(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }

// Density at the clamped voxel (i, j, k), substrate s, read as the reference
// reads it (motility.cpp:68-74: linear index voxel * S + s into the
// substrate-major buffer) or substrate-major.
__device__ __forceinline__ double dens_at(const DensView& d, int i, int j, int k, int s, int layout)
{
    i = clampi(i, static_cast<int>(d.nx) - 1);
    j = clampi(j, static_cast<int>(d.ny) - 1);
    k = clampi(k, static_cast<int>(d.nz) - 1);
    const uint64_t nvox = static_cast<uint64_t>(d.nx) * d.ny * d.nz;
    const uint64_t v = (static_cast<uint64_t>(k) * d.ny + j) * d.nx + i;
    const uint64_t lin = layout == PCG_MOT_REFERENCE ? v * d.S + s : static_cast<uint64_t>(s) * nvox + v;
    const uint64_t sub = lin / nvox, vv = lin % nvox;
    return static_cast<double>(d.base[sub * d.sub_pitch + (vv / d.nx) * d.px + vv % d.nx]);
}

// computeGradient (motility.cpp:46-87).  A substrate index outside
// [0, S) reads nothing and gives a zero gradient (the reference leaves it
// undefined).
__device__ void gradient(const DensView& d, float px, float py, float pz, int s, int layout, double& gx, double& gy,
                         double& gz)
{
    if (s < 0 || s >= static_cast<int>(d.S)) {
        gx = gy = gz = 0.0;
        return;
    }
    const int ix = clampi(static_cast<int>(__float2int_rz(__fdiv_rn(__fsub_rn(px, d.x_min), d.dx))),
                          static_cast<int>(d.nx) - 1);
    const int iy = clampi(static_cast<int>(__float2int_rz(__fdiv_rn(__fsub_rn(py, d.y_min), d.dy))),
                          static_cast<int>(d.ny) - 1);
    const int iz = clampi(static_cast<int>(__float2int_rz(__fdiv_rn(__fsub_rn(pz, d.z_min), d.dz))),
                          static_cast<int>(d.nz) - 1);
    gx = __ddiv_rn(__dsub_rn(dens_at(d, ix + 1, iy, iz, s, layout), dens_at(d, ix - 1, iy, iz, s, layout)),
                   2.0 * static_cast<double>(d.dx));
    gy = __ddiv_rn(__dsub_rn(dens_at(d, ix, iy + 1, iz, s, layout), dens_at(d, ix, iy - 1, iz, s, layout)),
                   2.0 * static_cast<double>(d.dy));
    gz = 0.0;
    if (d.nz > 1)
        gz = __ddiv_rn(__dsub_rn(dens_at(d, ix, iy, iz + 1, s, layout), dens_at(d, ix, iy, iz - 1, s, layout)),
                       2.0 * static_cast<double>(d.dz));
}

__device__ __forceinline__ double norm3(double x, double y, double z)
{
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}

__global__ void k_motility(float* __restrict__ soa, uint32_t stride, MotState m, DensView dv, bool have_density,
                           double dt, uint64_t seed, uint64_t step, int layout)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    if (__float_as_uint(soa[static_cast<size_t>(F_IS_ALIVE) * stride + i]) == 0u) return;
    double* mvx = m.vec;
    double* mvy = m.vec + m.n;
    double* mvz = m.vec + 2ull * m.n;
    if (m.is_motile[i] == 0u) {
        mvx[i] = mvy[i] = mvz[i] = 0.0;
        return;
    }
    m.elapsed[i] = __dadd_rn(m.elapsed[i], dt);
    const double pt = m.persistence[i];
    const bool resample = (pt < dt) || (uniform(seed, i, step, 0) < __ddiv_rn(dt, pt));
    if (resample) {
        m.elapsed[i] = 0.0;
        double rx, ry, rz;
        const double theta = __dmul_rn(2.0 * kPi, uniform(seed, i, step, 1));
        if (m.restrict_2d[i]) {
            rx = cos(theta);
            ry = sin(theta);
            rz = 0.0;
        } else {
            const double phi = __dmul_rn(kPi, uniform(seed, i, step, 2));
            const double sin_phi = sin(phi);
            rx = __dmul_rn(sin_phi, cos(theta));
            ry = __dmul_rn(sin_phi, sin(theta));
            rz = cos(phi);
        }
        double bx = 0.0, by = 0.0, bz = 0.0;
        const double bias = m.bias[i];
        if (bias > 0.0 && have_density) {
            const float px = soa[static_cast<size_t>(F_POS_X) * stride + i];
            const float py = soa[static_cast<size_t>(F_POS_Y) * stride + i];
            const float pz = soa[static_cast<size_t>(F_POS_Z) * stride + i];
            if (m.sens && m.n_sens > 0) {
                for (uint32_t s = 0; s < m.n_sens; ++s) {
                    const double sens = m.sens[static_cast<size_t>(i) * m.n_sens + s];
                    if (fabs(sens) < 1e-16) continue;
                    double gx, gy, gz;
                    gradient(dv, px, py, pz, static_cast<int>(s), layout, gx, gy, gz);
                    bx = __dadd_rn(bx, __dmul_rn(sens, gx));
                    by = __dadd_rn(by, __dmul_rn(sens, gy));
                    bz = __dadd_rn(bz, __dmul_rn(sens, gz));
                }
            } else {
                double gx, gy, gz;
                gradient(dv, px, py, pz, m.chem_index[i], layout, gx, gy, gz);
                const double dir = static_cast<double>(m.chem_dir[i]);
                bx = __dmul_rn(dir, gx);
                by = __dmul_rn(dir, gy);
                bz = __dmul_rn(dir, gz);
            }
            const double bmag = norm3(bx, by, bz);
            if (bmag > 1e-16) {
                bx = __ddiv_rn(bx, bmag);
                by = __ddiv_rn(by, bmag);
                bz = __ddiv_rn(bz, bmag);
            }
        }
        const double omb = __dsub_rn(1.0, bias);
        double mx = __dadd_rn(__dmul_rn(omb, rx), __dmul_rn(bias, bx));
        double my = __dadd_rn(__dmul_rn(omb, ry), __dmul_rn(bias, by));
        double mz = __dadd_rn(__dmul_rn(omb, rz), __dmul_rn(bias, bz));
        const double mag = norm3(mx, my, mz);
        if (mag > 1e-16) {
            mx = __ddiv_rn(mx, mag);
            my = __ddiv_rn(my, mag);
            mz = __ddiv_rn(mz, mag);
        }
        const double sp = static_cast<double>(soa[static_cast<size_t>(F_MOT_SPEED) * stride + i]);
        mvx[i] = __dmul_rn(mx, sp);
        mvy[i] = __dmul_rn(my, sp);
        mvz[i] = __dmul_rn(mz, sp);
    }
    float* v = soa + static_cast<size_t>(F_VEL_X) * stride + i;
    v[0] = __fadd_rn(v[0], static_cast<float>(mvx[i]));
    v[stride] = __fadd_rn(v[stride], static_cast<float>(mvy[i]));
    v[2ull * stride] = __fadd_rn(v[2ull * stride], static_cast<float>(mvz[i]));
}

}  // namespace

}  // namespace pcg

using namespace pcg;

struct pcg_motility {
    pcg_ctx* ctx = nullptr;
    uint32_t max_cells = 0, n_sens = 0, n = 0;
    DevBuf persistence, elapsed, bias, vec, is_motile, restrict_2d, chem_index, chem_dir, sens;
};

extern "C" {

pcg_status pcg_motility_create(pcg_ctx* ctx, uint32_t max_cells, uint32_t n_substrates, pcg_motility** out)
{
    if (!ctx || !out) return PCG_ERR_INVALID;
    *out = nullptr;
    if (max_cells == 0) return fail(ctx, PCG_ERR_INVALID, "max_cells must be >= 1");
    AllocStream pool_scope(ctx->stream);
    pcg_motility* m = new (std::nothrow) pcg_motility();
    if (!m) return PCG_ERR_OOM;
    m->ctx = ctx;
    m->max_cells = max_cells;
    m->n_sens = n_substrates;
    const size_t n = max_cells;
    cudaError_t e = cudaSuccess;
    for (DevBuf* b : {&m->persistence, &m->elapsed, &m->bias})
        if (e == cudaSuccess) e = b->alloc(n * sizeof(double));
    if (e == cudaSuccess) e = m->vec.alloc(3 * n * sizeof(double));
    for (DevBuf* b : {&m->is_motile, &m->restrict_2d, &m->chem_index, &m->chem_dir})
        if (e == cudaSuccess) e = b->alloc(n * sizeof(uint32_t));
    if (e == cudaSuccess && n_substrates) e = m->sens.alloc(n * n_substrates * sizeof(double));
    if (e != cudaSuccess) {
        delete m;
        return cuda_fail(ctx, e, "motility allocation");
    }
    ctx_retain(ctx);
    *out = m;
    return PCG_OK;
}

pcg_status pcg_motility_destroy(pcg_motility* m)
{
    if (!m) return PCG_ERR_INVALID;
    pcg_ctx* ctx = m->ctx;
    delete m;
    ctx_release(ctx);
    return PCG_OK;
}

pcg_status pcg_motility_upload(pcg_motility* m, uint32_t n, const double* persistence, const double* elapsed,
                               const double* bias, const double* vec, const uint32_t* is_motile,
                               const uint32_t* restrict_2d, const int32_t* chem_index, const int32_t* chem_dir,
                               const double* sensitivity)
{
    if (!m) return PCG_ERR_INVALID;
    pcg_ctx* ctx = m->ctx;
    if (n > m->max_cells) return fail(ctx, PCG_ERR_INVALID, "n_cells exceeds max_cells");
    if (!persistence || !elapsed || !bias || !vec || !is_motile || !restrict_2d || !chem_index || !chem_dir)
        return fail(ctx, PCG_ERR_INVALID, "null motility array");
    if (m->n_sens && !sensitivity) return fail(ctx, PCG_ERR_INVALID, "sensitivity required (created with substrates)");
    m->n = n;
    if (n == 0) return PCG_OK;
    cudaStream_t st = ctx->stream;
    const size_t d = static_cast<size_t>(n) * sizeof(double), u = static_cast<size_t>(n) * sizeof(uint32_t);
    PCG_CU(ctx, cudaMemcpyAsync(m->persistence.p, persistence, d, cudaMemcpyHostToDevice, st));
    PCG_CU(ctx, cudaMemcpyAsync(m->elapsed.p, elapsed, d, cudaMemcpyHostToDevice, st));
    PCG_CU(ctx, cudaMemcpyAsync(m->bias.p, bias, d, cudaMemcpyHostToDevice, st));
    for (int a = 0; a < 3; ++a)   // host x, y, z arrays of n -> device arrays of n (packed)
        PCG_CU(ctx, cudaMemcpyAsync(m->vec.as<double>() + static_cast<size_t>(a) * n, vec + static_cast<size_t>(a) * n, d,
                                    cudaMemcpyHostToDevice, st));
    PCG_CU(ctx, cudaMemcpyAsync(m->is_motile.p, is_motile, u, cudaMemcpyHostToDevice, st));
    PCG_CU(ctx, cudaMemcpyAsync(m->restrict_2d.p, restrict_2d, u, cudaMemcpyHostToDevice, st));
    PCG_CU(ctx, cudaMemcpyAsync(m->chem_index.p, chem_index, u, cudaMemcpyHostToDevice, st));
    PCG_CU(ctx, cudaMemcpyAsync(m->chem_dir.p, chem_dir, u, cudaMemcpyHostToDevice, st));
    if (m->n_sens)
        PCG_CU(ctx, cudaMemcpyAsync(m->sens.p, sensitivity, d * m->n_sens, cudaMemcpyHostToDevice, st));
    PCG_CU(ctx, cudaStreamSynchronize(st));   // the caller may reuse its arrays on return
    return PCG_OK;
}

pcg_status pcg_motility_download(pcg_motility* m, double* elapsed, double* vec)
{
    if (!m) return PCG_ERR_INVALID;
    pcg_ctx* ctx = m->ctx;
    const size_t n = m->n, d = n * sizeof(double);
    if (n) {
        if (elapsed) PCG_CU(ctx, cudaMemcpyAsync(elapsed, m->elapsed.p, d, cudaMemcpyDeviceToHost, ctx->stream));
        if (vec) PCG_CU(ctx, cudaMemcpyAsync(vec, m->vec.p, 3 * d, cudaMemcpyDeviceToHost, ctx->stream));
    }
    PCG_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return PCG_OK;
}

pcg_status pcg_motility_update(pcg_motility* m, pcg_cells* cells, const pcg_me* me, double dt, uint64_t seed,
                               uint64_t step, int layout)
{
    if (!m || !cells) return PCG_ERR_INVALID;
    pcg_ctx* ctx = m->ctx;
    if (cells->ctx != ctx || (me && me->ctx != ctx)) return fail(ctx, PCG_ERR_INVALID, "objects of different contexts");
    if (layout != PCG_MOT_REFERENCE && layout != PCG_MOT_SUBSTRATE_MAJOR) return fail(ctx, PCG_ERR_INVALID, "bad layout");
    if (m->n > cells->c.n) return fail(ctx, PCG_ERR_INVALID, "motility state covers more cells than the cell store");
    if (m->n == 0) return PCG_OK;
    DensView dv{};
    const bool have = me != nullptr;
    if (have) {
        const DiffInstance& di = me->d.inst[0];
        const pcg_grid_params& g = di.g;
        if (m->n_sens && m->n_sens != g.n_substrates)
            return fail(ctx, PCG_ERR_INVALID, "sensitivity substrates differ from the microenvironment's");
        dv.base = me->d.dens.as<float>() + di.dens_off;
        dv.sub_pitch = di.pitch;
        dv.px = di.px;
        dv.nx = g.nx;
        dv.ny = g.ny;
        dv.nz = g.nz;
        dv.S = g.n_substrates;
        dv.dx = g.dx;
        dv.dy = g.dy;
        dv.dz = g.dz;
        dv.x_min = g.x_min;
        dv.y_min = g.y_min;
        dv.z_min = g.z_min;
    }
    MotState ms{m->persistence.as<double>(), m->elapsed.as<double>(), m->bias.as<double>(), m->vec.as<double>(),
                m->is_motile.as<uint32_t>(), m->restrict_2d.as<uint32_t>(), m->chem_index.as<int32_t>(),
                m->chem_dir.as<int32_t>(), m->n_sens ? m->sens.as<double>() : nullptr, m->n_sens, m->n};
    const unsigned grid = (m->n + 127) / 128;
    k_motility<<<grid, 128, 0, ctx->stream>>>(cells->c.soa.as<float>(), cells->c.max_cells, ms, dv, have, dt, seed,
                                              step, layout);
    PCG_CU(ctx, cudaGetLastError());
    ctx->launches++;
    return PCG_OK;
}

}  // extern "C"
