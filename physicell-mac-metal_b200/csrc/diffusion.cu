// diffusion.cu — LOD Thomas sweeps, Dirichlet reset and gradients (sm_100a).
//
// Reference semantics: shaders/diffusion_2d.metal:28-157 (x sweep) and
// :165-292 (y sweep), one tridiagonal solve per line over the interior
// nodes 1..n-2 with the decay on the diagonal; src/microenvironment.mm:212-237
// (applyDirichletBC); :282-342 (computeGradients).  The z sweep applies the
// same per-line rule along k.
//
// The solve.  Every line of one (instance, substrate, axis) family has the
// same matrix, so g_i = c / den_i and 1 / den_i are one table (LineRule,
// built in FP64 on the host).  With h_i = (rho_i + fold_i) / den_i the
// reference's forward and backward passes are two first-order linear
// recurrences with the same coefficients:
//     forward   d_i = g_i d_{i-1} + h_i        (d_0 = 0)
//     backward  x_i = g_i x_{i+1} + d_i        (x_{n-1} = 0)
// End nodes (and padding) have g = h = 0, so they are transparent; they
// keep their value, or take the Dirichlet target.  A line is cut into
// chunks held in registers: each thread runs both recurrences over its
// chunk, and the chunks are joined by an exclusive scan of affine maps
// (x -> A x + B), forward for d and in reverse for x.  Every value is read
// from HBM once and written once per sweep; nothing is staged in shared
// memory except the per-chunk maps of the y/z scan.
//   x sweep   a segment of S = 8/16/32 lanes of one warp per line (the line
//             is contiguous), chunks of m = ceil(n / S) values, scan with
//             warp shuffles;
//   y/z sweep lanes are 32 adjacent columns (each row a 128-byte segment),
//             the 16 warps of a CTA are chunks along the line, scan through
//             shared memory.
// The chunking depends only on the line length, so a line's arithmetic is
// the same whatever else shares the launch.
#include "pcg_kernels.cuh"

namespace pcg {

__device__ __forceinline__ bool tile_on(const LineRule& r, const uint8_t* __restrict__ mask)
{
    return mask == nullptr || (mask[r.inst] & STEP_DIFFUSE);
}

__device__ __forceinline__ bool on_face(const SweepTile& tile, int lane)
{
    if (tile.face & TILE_FACE_ALL) return true;
    const uint32_t i = tile.i0 + static_cast<uint32_t>(lane);
    return i == 0u || i + 1u == tile.nx;
}

// Reference rule for a whole line held at s[m * st] (used for lines too long
// for the chunked kernels): the same recurrences, sequentially.
__device__ __forceinline__ void solve_line(float* s, int st, const LineRule& r, const float2* __restrict__ tb)
{
    const int n = static_cast<int>(r.n);
    if (n >= 3) {
        float d = 0.f;
        for (int i = 1; i <= n - 2; ++i) {
            const float2 e = __ldg(&tb[i]);
            const float f = (i == 1 || i == n - 2) ? r.fold : 0.f;
            d = fmaf(-e.x, d, (s[i * st] + f) * e.y);
            s[i * st] = d;
        }
        float x = 0.f;
        for (int i = n - 2; i >= 1; --i) {
            x = fmaf(-__ldg(&tb[i].x), x, s[i * st]);
            s[i * st] = x;
        }
    }
    if (r.dir) {
        s[0] = r.T;
        s[(n - 1) * st] = r.T;
    }
}

// ------------------------------------------------------------------ x sweep

template <int M>
__global__ void __launch_bounds__(256) k_sweep_x(float* __restrict__ dens, const SweepTile* __restrict__ tiles,
                                                 uint32_t ntiles, const LineRule* __restrict__ rules,
                                                 const float2* __restrict__ tab, const uint8_t* __restrict__ mask)
{
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = gw; t < ntiles; t += nw) {
        const SweepTile tile = tiles[t];
        const LineRule r = rules[tile.rule];
        if (!tile_on(r, mask)) continue;
        const int n = static_cast<int>(r.n);
        const int S = static_cast<int>(x_seg_lanes(r.n));
        const int m = (n + S - 1) / S;
        const int seg = lane / S, sl = lane % S;
        const bool active = seg < static_cast<int>(tile.count);
        float* g = dens + tile.base + static_cast<size_t>(seg) * n;
        const float2* tb = tab + r.tab;
        const int p0 = sl * m;
        float v[M], gg[M];
#pragma unroll
        for (int k = 0; k < M; ++k) {
            const int p = p0 + k;
            float x = 0.f, gk = 0.f, iv = 0.f;
            if (k < m && active && p < n) {
                x = g[p];
                const float2 e = __ldg(&tb[p]);
                gk = -e.x;
                iv = e.y;
            }
            const float f = (p == 1 || p == n - 2) ? r.fold : 0.f;
            v[k] = (x + f) * iv;
            gg[k] = gk;
        }
        // forward: local recurrence, then the segment's exclusive scan
        float d = 0.f, A = 1.f;
#pragma unroll
        for (int k = 0; k < M; ++k) {
            if (k < m) {
                d = fmaf(gg[k], d, v[k]);
                A *= gg[k];
                v[k] = d;
            }
        }
        float B = d;
        for (int o = 1; o < S; o <<= 1) {
            const float Ap = __shfl_up_sync(0xffffffffu, A, o, S);
            const float Bp = __shfl_up_sync(0xffffffffu, B, o, S);
            if (sl >= o) {
                B = fmaf(A, Bp, B);
                A *= Ap;
            }
        }
        float din = __shfl_up_sync(0xffffffffu, B, 1, S);
        if (sl == 0) din = 0.f;
        float run = 1.f;
#pragma unroll
        for (int k = 0; k < M; ++k) {
            if (k < m) {
                run *= gg[k];
                v[k] = fmaf(run, din, v[k]);
            }
        }
        // backward: local recurrence from the chunk's end, reverse scan
        float x = 0.f;
        A = 1.f;
#pragma unroll
        for (int k = M - 1; k >= 0; --k) {
            if (k < m) {
                x = fmaf(gg[k], x, v[k]);
                A *= gg[k];
                v[k] = x;
            }
        }
        B = x;
        for (int o = 1; o < S; o <<= 1) {
            const float Ap = __shfl_down_sync(0xffffffffu, A, o, S);
            const float Bp = __shfl_down_sync(0xffffffffu, B, o, S);
            if (sl + o < S) {
                B = fmaf(A, Bp, B);
                A *= Ap;
            }
        }
        float xout = __shfl_down_sync(0xffffffffu, B, 1, S);
        if (sl == S - 1) xout = 0.f;
        run = 1.f;
#pragma unroll
        for (int k = M - 1; k >= 0; --k) {
            if (k < m) {
                run *= gg[k];
                v[k] = fmaf(run, xout, v[k]);
            }
        }
        if (active) {
#pragma unroll
            for (int k = 0; k < M; ++k) {
                const int p = p0 + k;
                if (k < m && p < n) {
                    if (p == 0 || p == n - 1) {
                        if (r.dir) g[p] = r.T;
                    } else {
                        g[p] = v[k];
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------- y/z sweeps

constexpr int kColsWarps = 16;

template <int M>
__global__ void __launch_bounds__(kColsWarps * 32) k_sweep_cols(float* __restrict__ dens,
                                                                const SweepTile* __restrict__ tiles, uint32_t ntiles,
                                                                const LineRule* __restrict__ rules,
                                                                const float2* __restrict__ tab, int apply_faces,
                                                                const uint8_t* __restrict__ mask)
{
    __shared__ float sA[kColsWarps][32], sB[kColsWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const SweepTile tile = tiles[t];
        const LineRule r = rules[tile.rule];
        if (!tile_on(r, mask)) continue;   // uniform over the CTA
        const int n = static_cast<int>(r.n);
        const int m = static_cast<int>(cols_chunk(r.n));
        const int W = (n + m - 1) / m;
        const bool col_ok = lane < static_cast<int>(tile.count);
        const bool face = apply_faces && (tile.face & TILE_FACE) && on_face(tile, lane);
        const bool work = col_ok && !face && w < W;
        float* col = dens + tile.base + lane;
        const size_t rs = tile.rs;
        const float2* tb = tab + r.tab;
        const int p0 = w * m;
        float v[M], gg[M];
#pragma unroll
        for (int k = 0; k < M; ++k) {
            const int p = p0 + k;
            float x = 0.f, gk = 0.f, iv = 0.f;
            if (k < m && work && p < n) {
                x = col[p * rs];
                const float2 e = __ldg(&tb[p]);
                gk = -e.x;
                iv = e.y;
            }
            const float f = (p == 1 || p == n - 2) ? r.fold : 0.f;
            v[k] = (x + f) * iv;
            gg[k] = gk;
        }
        float d = 0.f, A = 1.f;
#pragma unroll
        for (int k = 0; k < M; ++k) {
            if (k < m) {
                d = fmaf(gg[k], d, v[k]);
                A *= gg[k];
                v[k] = d;
            }
        }
        sA[w][lane] = A;
        sB[w][lane] = d;
        __syncthreads();
        float din = 0.f;
        for (int q = 0; q < w && q < W; ++q) din = fmaf(sA[q][lane], din, sB[q][lane]);
        __syncthreads();
        float run = 1.f;
#pragma unroll
        for (int k = 0; k < M; ++k) {
            if (k < m) {
                run *= gg[k];
                v[k] = fmaf(run, din, v[k]);
            }
        }
        float x = 0.f;
        A = 1.f;
#pragma unroll
        for (int k = M - 1; k >= 0; --k) {
            if (k < m) {
                x = fmaf(gg[k], x, v[k]);
                A *= gg[k];
                v[k] = x;
            }
        }
        sA[w][lane] = A;
        sB[w][lane] = x;
        __syncthreads();
        float xout = 0.f;
        for (int q = W - 1; q > w; --q) xout = fmaf(sA[q][lane], xout, sB[q][lane]);
        run = 1.f;
#pragma unroll
        for (int k = M - 1; k >= 0; --k) {
            if (k < m) {
                run *= gg[k];
                v[k] = fmaf(run, xout, v[k]);
            }
        }
        if (col_ok && w < W) {
#pragma unroll
            for (int k = 0; k < M; ++k) {
                const int p = p0 + k;
                if (k < m && p < n) {
                    if (face) {
                        col[p * rs] = r.T;   // applyDirichletBC fused: the line lies on a face
                    } else if (p == 0 || p == n - 1) {
                        if (r.dir) col[p * rs] = r.T;
                    } else {
                        col[p * rs] = v[k];
                    }
                }
            }
        }
        __syncthreads();
    }
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

template <int M>
static int occ_x(int block)
{
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sweep_x<M>, block, 0) != cudaSuccess) return 0;
    return b;
}
template <int M>
static int occ_cols()
{
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sweep_cols<M>, kColsWarps * 32, 0) != cudaSuccess)
        return 0;
    return b;
}

int sweep_x_occupancy(int nmax, int block)
{
    switch (x_chunk_template(static_cast<uint32_t>(nmax))) {
        case 4: return occ_x<4>(block);
        case 8: return occ_x<8>(block);
        case 16: return occ_x<16>(block);
        default: return 0;
    }
}

int sweep_cols_occupancy(int nmax)
{
    switch (cols_chunk_template(static_cast<uint32_t>(nmax))) {
        case 8: return occ_cols<8>();
        case 16: return occ_cols<16>();
        case 32: return occ_cols<32>();
        default: return 0;
    }
}

cudaError_t launch_sweep_x(cudaStream_t st, float* dens, const SweepTile* tiles, uint32_t ntiles,
                           const LineRule* rules, const float2* tab, int nmax, const uint8_t* mask, RowsCfg cfg)
{
    if (ntiles == 0) return cudaSuccess;
    switch (x_chunk_template(static_cast<uint32_t>(nmax))) {
        case 4: k_sweep_x<4><<<cfg.grid, cfg.block, 0, st>>>(dens, tiles, ntiles, rules, tab, mask); break;
        case 8: k_sweep_x<8><<<cfg.grid, cfg.block, 0, st>>>(dens, tiles, ntiles, rules, tab, mask); break;
        case 16: k_sweep_x<16><<<cfg.grid, cfg.block, 0, st>>>(dens, tiles, ntiles, rules, tab, mask); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_sweep_cols(cudaStream_t st, float* dens, const SweepTile* tiles, uint32_t ntiles,
                              const LineRule* rules, const float2* tab, int nmax, int apply_faces,
                              const uint8_t* mask, ColsCfg cfg)
{
    if (ntiles == 0) return cudaSuccess;
    const int b = kColsWarps * 32;
    switch (cols_chunk_template(static_cast<uint32_t>(nmax))) {
        case 8: k_sweep_cols<8><<<cfg.grid, b, 0, st>>>(dens, tiles, ntiles, rules, tab, apply_faces, mask); break;
        case 16: k_sweep_cols<16><<<cfg.grid, b, 0, st>>>(dens, tiles, ntiles, rules, tab, apply_faces, mask); break;
        case 32: k_sweep_cols<32><<<cfg.grid, b, 0, st>>>(dens, tiles, ntiles, rules, tab, apply_faces, mask); break;
        default: return cudaErrorInvalidValue;
    }
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
