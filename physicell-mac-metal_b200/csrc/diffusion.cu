// diffusion.cu — LOD Thomas sweeps, Dirichlet reset and gradients (sm_100a).
//
// Reference semantics: shaders/diffusion_2d.metal:28-157 (x sweep) and
// :165-292 (y sweep), one tridiagonal solve per line over the interior
// nodes 1..n-2 with the decay on the diagonal; src/microenvironment.mm:212-237
// (applyDirichletBC); :282-342 (computeGradients).  The z sweep applies the
// same per-line rule along k.
//
// B200 layout.  density is [s][k][j][i] FP32 in HBM.  The per-line Thomas
// constants are one table per (instance, substrate, axis) (LineRule), so the
// forward pass is one FMUL + one FFMA per value and the backward pass one
// FFMA.  Work is a flat list of tiles over all instances:
//   x sweep   row tiles: L contiguous lines (one CTA, one line per thread),
//             staged through padded shared memory (stride n|1, conflict-free)
//             with cp.async, double-buffered across tiles;
//   y/z sweep column tiles: 32 adjacent columns (one warp, one column per
//             lane), each row a 128-byte coalesced segment, staged with
//             cp.async, double-buffered per warp.
// Each value is read from HBM once and written once per sweep.
#include "pcg_kernels.cuh"

namespace pcg {

__device__ __forceinline__ void cp_async4(float* smem, const float* gmem)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Solve one line in place; s[m * st] is position m.  Implements the rule of
// diffusion_2d.metal:55-155 with the precomputed table (see LineRule).
__device__ __forceinline__ void solve_line(float* s, int st, const LineRule& r, const float2* __restrict__ tb)
{
    const int n = static_cast<int>(r.n);
    if (n >= 3) {
        const float f = r.fold;
        if (n == 3) {
            s[st] = (s[st] + f) * __ldg(&tb[1].y);
        } else {
            float d = (s[st] + f) * __ldg(&tb[1].y);
            s[st] = d;
            int i = 2;
#pragma unroll 4
            for (; i < n - 2; ++i) {
                const float2 e = __ldg(&tb[i]);
                d = fmaf(-e.x, d, s[i * st] * e.y);
                s[i * st] = d;
            }
            {
                const float2 e = __ldg(&tb[n - 2]);
                d = fmaf(-e.x, d, (s[(n - 2) * st] + f) * e.y);
                s[(n - 2) * st] = d;
            }
#pragma unroll 4
            for (i = n - 3; i >= 1; --i) {
                d = fmaf(-__ldg(&tb[i].x), d, s[i * st]);
                s[i * st] = d;
            }
        }
    }
    if (r.dir) {
        s[0] = r.T;
        s[(n - 1) * st] = r.T;
    }
}

// ------------------------------------------------------------------ x sweep

__device__ __forceinline__ void rows_issue(const SweepTile& tile, const LineRule* __restrict__ rules,
                                           const float* __restrict__ dens, float* buf)
{
    const uint32_t n = rules[tile.rule].n;
    const uint32_t P = n | 1u;
    const uint32_t total = tile.count * n;
    const float* g = dens + tile.base;
    const uint32_t M = (n == 1u) ? 0u : (0xFFFFFFFFu / n + 1u);   // ceil(2^32 / n)
    for (uint32_t e = threadIdx.x; e < total; e += blockDim.x) {
        const uint32_t line = (n == 1u) ? e : __umulhi(e, M);
        const uint32_t pos = e - line * n;
        cp_async4(buf + line * P + pos, g + e);
    }
}

__device__ __forceinline__ bool tile_on(const LineRule& r, const uint8_t* __restrict__ mask)
{
    return mask == nullptr || (mask[r.inst] & STEP_DIFFUSE);
}

__global__ void __launch_bounds__(256) k_sweep_rows(float* __restrict__ dens, const SweepTile* __restrict__ tiles,
                                                    uint32_t ntiles, const LineRule* __restrict__ rules,
                                                    const float2* __restrict__ tab, int pmax,
                                                    const uint8_t* __restrict__ mask)
{
    extern __shared__ float sm[];
    float* bufs[2] = {sm, sm + static_cast<size_t>(blockDim.x) * pmax};
    uint32_t t = blockIdx.x;
    if (t < ntiles) rows_issue(tiles[t], rules, dens, bufs[0]);
    cp_async_commit();
    int k = 0;
    for (; t < ntiles; t += gridDim.x, k ^= 1) {
        const uint32_t tn = t + gridDim.x;
        if (tn < ntiles) rows_issue(tiles[tn], rules, dens, bufs[k ^ 1]);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const SweepTile tile = tiles[t];
        const LineRule r = rules[tile.rule];
        const uint32_t n = r.n, P = n | 1u, total = tile.count * n;
        float* buf = bufs[k];
        if (!tile_on(r, mask)) {
            __syncthreads();
            continue;
        }
        if (threadIdx.x < tile.count) solve_line(buf + threadIdx.x * P, 1, r, tab + r.tab);
        __syncthreads();
        float* g = dens + tile.base;
        const uint32_t M = (n == 1u) ? 0u : (0xFFFFFFFFu / n + 1u);
        for (uint32_t e = threadIdx.x; e < total; e += blockDim.x) {
            const uint32_t line = (n == 1u) ? e : __umulhi(e, M);
            g[e] = buf[line * P + (e - line * n)];
        }
        __syncthreads();
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------- y/z sweeps

__device__ __forceinline__ void cols_issue(const SweepTile& tile, const LineRule* __restrict__ rules,
                                           const float* __restrict__ dens, float* buf, int lane)
{
    if (static_cast<uint32_t>(lane) >= tile.count) return;
    const uint32_t n = rules[tile.rule].n;
    const float* g = dens + tile.base + lane;
    const size_t rs = tile.rs;
    for (uint32_t j = 0; j < n; ++j) cp_async4(buf + j * 32 + lane, g + j * rs);
}

__device__ __forceinline__ bool on_face(const SweepTile& tile, int lane)
{
    if (tile.face & TILE_FACE_ALL) return true;
    const uint32_t i = tile.i0 + static_cast<uint32_t>(lane);
    return i == 0u || i + 1u == tile.nx;
}

__global__ void __launch_bounds__(256) k_sweep_cols(float* __restrict__ dens, const SweepTile* __restrict__ tiles,
                                                    uint32_t ntiles, const LineRule* __restrict__ rules,
                                                    const float2* __restrict__ tab, int nmax, int apply_faces,
                                                    const uint8_t* __restrict__ mask)
{
    extern __shared__ float sm[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    float* bufs[2];
    bufs[0] = sm + static_cast<size_t>(warp) * 2 * nmax * 32;
    bufs[1] = bufs[0] + static_cast<size_t>(nmax) * 32;
    const uint32_t step = gridDim.x * wpb;
    uint32_t t = blockIdx.x * wpb + warp;
    if (t < ntiles) cols_issue(tiles[t], rules, dens, bufs[0], lane);
    cp_async_commit();
    int k = 0;
    for (; t < ntiles; t += step, k ^= 1) {
        const uint32_t tn = t + step;
        if (tn < ntiles) cols_issue(tiles[tn], rules, dens, bufs[k ^ 1], lane);
        cp_async_commit();
        cp_async_wait<1>();
        const SweepTile tile = tiles[t];
        const LineRule r = rules[tile.rule];
        if (static_cast<uint32_t>(lane) < tile.count && tile_on(r, mask)) {
            const int n = static_cast<int>(r.n);
            float* col = bufs[k] + lane;
            float* g = dens + tile.base + lane;
            const size_t rs = tile.rs;
            if (apply_faces && (tile.face & TILE_FACE) && on_face(tile, lane)) {
                // applyDirichletBC fused: the whole line lies on a Dirichlet face
                for (int j = 0; j < n; ++j) g[j * rs] = r.T;
            } else {
                solve_line(col, 32, r, tab + r.tab);
                for (int j = 0; j < n; ++j) g[j * rs] = col[j * 32];
            }
        }
    }
    cp_async_wait<0>();
}

// ------------------------------------------------------- any line length

__global__ void __launch_bounds__(128) k_sweep_global(float* __restrict__ dens, const SweepTile* __restrict__ tiles,
                                                      uint32_t ntiles, const LineRule* __restrict__ rules,
                                                      const float2* __restrict__ tab, int apply_faces,
                                                      const uint8_t* __restrict__ mask)
{
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = gw; t < ntiles; t += nw) {
        const SweepTile tile = tiles[t];
        if (static_cast<uint32_t>(lane) >= tile.count) continue;
        const LineRule r = rules[tile.rule];
        if (!tile_on(r, mask)) continue;
        const uint32_t ls = tile.rs == 1u ? r.n : 1u;
        float* g = dens + tile.base + static_cast<size_t>(lane) * ls;
        if (apply_faces && (tile.face & TILE_FACE) && on_face(tile, lane)) {
            for (uint32_t j = 0; j < r.n; ++j) g[static_cast<size_t>(j) * tile.rs] = r.T;
        } else {
            solve_line(g, static_cast<int>(tile.rs), r, tab + r.tab);
        }
    }
}

// ------------------------------------------------------------- Dirichlet

__global__ void k_dirichlet(float* __restrict__ dens, const FaceJob* __restrict__ jobs)
{
    const FaceJob jb = jobs[blockIdx.x];
    float* base = dens + jb.base;
    const uint32_t nx = jb.nx, ny = jb.ny, nz = jb.nz;
    const size_t slab = static_cast<size_t>(nx) * ny;
    // edges of every slab (microenvironment.mm:225-235)
    const uint32_t per = 2u * nx + 2u * ny;
    const size_t total = static_cast<size_t>(nz) * per;
    for (size_t e = threadIdx.x; e < total; e += blockDim.x) {
        const uint32_t k = static_cast<uint32_t>(e / per), q = static_cast<uint32_t>(e % per);
        uint32_t i, j;
        if (q < nx) { i = q; j = 0; }
        else if (q < 2u * nx) { i = q - nx; j = ny - 1; }
        else if (q < 2u * nx + ny) { i = 0; j = q - 2u * nx; }
        else { i = nx - 1; j = q - 2u * nx - ny; }
        base[k * slab + static_cast<size_t>(j) * nx + i] = jb.T;
    }
    if (nz > 1) {   // z faces (3-D rule)
        for (size_t e = threadIdx.x; e < 2 * slab; e += blockDim.x) {
            const size_t k = (e < slab) ? 0 : (nz - 1);
            base[k * slab + (e % slab)] = jb.T;
        }
    }
}

// ------------------------------------------------------------- gradients

__global__ void k_gradients(const float* __restrict__ dens, float* __restrict__ gx, float* __restrict__ gy,
                            float* __restrict__ gz, const GradJob* __restrict__ jobs)
{
    const GradJob jb = jobs[blockIdx.y];
    const size_t nx = jb.nx, ny = jb.ny, nz = jb.nz, nv = nx * ny * nz;
    const float* D = dens + jb.base;
    for (size_t n = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; n < nv;
         n += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t i = n % nx, j = (n / nx) % ny, k = n / (nx * ny);
        const size_t o = jb.out_base + n;
        double v;
        if (nx == 1) v = 0.0;
        else if (i == 0) v = (static_cast<double>(D[n + 1]) - D[n]) * jb.inv_dx;
        else if (i == nx - 1) v = (static_cast<double>(D[n]) - D[n - 1]) * jb.inv_dx;
        else v = (static_cast<double>(D[n + 1]) - D[n - 1]) * 0.5 * jb.inv_dx;
        if (gx) gx[o] = static_cast<float>(v);
        if (ny == 1) v = 0.0;
        else if (j == 0) v = (static_cast<double>(D[n + nx]) - D[n]) * jb.inv_dy;
        else if (j == ny - 1) v = (static_cast<double>(D[n]) - D[n - nx]) * jb.inv_dy;
        else v = (static_cast<double>(D[n + nx]) - D[n - nx]) * 0.5 * jb.inv_dy;
        if (gy) gy[o] = static_cast<float>(v);
        if (nz > 1) {
            const size_t sz = nx * ny;
            if (k == 0) v = (static_cast<double>(D[n + sz]) - D[n]) * jb.inv_dz;
            else if (k == nz - 1) v = (static_cast<double>(D[n]) - D[n - sz]) * jb.inv_dz;
            else v = (static_cast<double>(D[n + sz]) - D[n - sz]) * 0.5 * jb.inv_dz;
        } else {
            v = 0.0;
        }
        if (gz) gz[o] = static_cast<float>(v);
    }
}

// ------------------------------------------------------------- launchers

size_t sweep_rows_smem(int lines, int nmax) { return 2u * static_cast<size_t>(lines) * (nmax | 1) * sizeof(float); }
size_t sweep_cols_smem(int warps, int nmax) { return 2u * static_cast<size_t>(warps) * nmax * 32 * sizeof(float); }

// The attribute is per kernel, shared by every object in the process, so it
// is always raised to the device's opt-in maximum (never lowered).
static cudaError_t allow_max_smem(const void* fn)
{
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    return e;
}
cudaError_t sweep_rows_prepare(int lines, int nmax)
{
    if (sweep_rows_smem(lines, nmax) > 232448) return cudaErrorInvalidValue;
    return allow_max_smem(reinterpret_cast<const void*>(k_sweep_rows));
}
cudaError_t sweep_cols_prepare(int warps, int nmax)
{
    if (sweep_cols_smem(warps, nmax) > 232448) return cudaErrorInvalidValue;
    return allow_max_smem(reinterpret_cast<const void*>(k_sweep_cols));
}
int sweep_rows_occupancy(int lines, int nmax)
{
    int b = 0;
    if (sweep_rows_prepare(lines, nmax) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sweep_rows, lines, sweep_rows_smem(lines, nmax)) !=
        cudaSuccess)
        return 0;
    return b;
}
int sweep_cols_occupancy(int warps, int nmax)
{
    int b = 0;
    if (sweep_cols_prepare(warps, nmax) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sweep_cols, warps * 32, sweep_cols_smem(warps, nmax)) !=
        cudaSuccess)
        return 0;
    return b;
}

cudaError_t launch_sweep_rows(cudaStream_t st, float* dens, const SweepTile* tiles, uint32_t ntiles,
                              const LineRule* rules, const float2* tab, int nmax, const uint8_t* mask, RowsCfg cfg)
{
    if (ntiles == 0) return cudaSuccess;
    const int pmax = nmax | 1;
    k_sweep_rows<<<cfg.grid, cfg.lines, sweep_rows_smem(cfg.lines, nmax), st>>>(dens, tiles, ntiles, rules, tab, pmax,
                                                                                  mask);
    return cudaGetLastError();
}

cudaError_t launch_sweep_cols(cudaStream_t st, float* dens, const SweepTile* tiles, uint32_t ntiles,
                              const LineRule* rules, const float2* tab, int nmax, int apply_faces,
                              const uint8_t* mask, ColsCfg cfg)
{
    if (ntiles == 0) return cudaSuccess;
    k_sweep_cols<<<cfg.grid, cfg.warps * 32, sweep_cols_smem(cfg.warps, nmax), st>>>(dens, tiles, ntiles, rules, tab,
                                                                                       nmax, apply_faces, mask);
    return cudaGetLastError();
}

cudaError_t launch_sweep_global(cudaStream_t st, float* dens, const SweepTile* tiles, uint32_t ntiles,
                                const LineRule* rules, const float2* tab, int apply_faces, const uint8_t* mask,
                                int grid)
{
    if (ntiles == 0) return cudaSuccess;
    k_sweep_global<<<grid, 128, 0, st>>>(dens, tiles, ntiles, rules, tab, apply_faces, mask);
    return cudaGetLastError();
}

cudaError_t launch_dirichlet(cudaStream_t st, float* dens, const FaceJob* jobs, uint32_t njobs)
{
    if (njobs == 0) return cudaSuccess;
    k_dirichlet<<<njobs, 256, 0, st>>>(dens, jobs);
    return cudaGetLastError();
}

cudaError_t launch_gradients(cudaStream_t st, const float* dens, float* gx, float* gy, float* gz,
                             const GradJob* jobs, uint32_t njobs, uint64_t max_voxels)
{
    if (njobs == 0) return cudaSuccess;
    uint64_t bx = (max_voxels + 255) / 256;
    if (bx > 4096) bx = 4096;
    if (bx == 0) bx = 1;
    dim3 grid(static_cast<unsigned>(bx), njobs);
    k_gradients<<<grid, 256, 0, st>>>(dens, gx, gy, gz, jobs);
    return cudaGetLastError();
}

}  // namespace pcg
