// secorder.cu — the secretion order (sm_100a): every instance's cells sorted
// by (diffusion voxel, cell index), rebuilt whenever voxel indices change
// (after every mechanics step when they are refreshed).
//
// processSecretion (cell_phenotype.cpp:526-564) runs cell by cell in the
// reference; the order of the cells that share a voxel decides the FP32
// roundings, so the device applies each voxel's cells in ascending index.
//
// The order is a stable LSD radix sort of each instance's cells on the
// cell's voxel index within its own grid (at most 21 bits for a 120^3 grid,
// so three passes of 7-bit digits), segmented by instance: tiles of 2048
// cells never straddle two instances, so every instance's cells stay in the
// instance's own range [cell_off, cell_off + n_cells) and the places of one
// instance's (digit, tile) runs depend on that instance's counts alone.
// A cell that takes no part in secretion (inactive, voxel index outside the
// grid, no substrates) has the extra digit R of every pass, so it ends up
// after the instance's secreting cells, in index order.
//
// One pass:
//   k_so_hist     per tile: digit counts, one row of R + 1 per tile (the
//                 first pass also computes the keys from the SoA and stores
//                 them in cell order)
//   k_so_offsets  per instance: digit totals over its tiles, their scan from
//                 cell_off, then each tile's row turned into the first place
//                 of each of its digit runs (digit-major, tiles in order)
//   k_so_scatter  per tile: stable ranks (each warp ranks its 256 keys with
//                 __match_any_sync and its own running digit counts, warps
//                 combined in order), the tile laid out in shared
//                 memory in digit order, then written so that consecutive
//                 threads store consecutive elements of one digit's run; the
//                 last pass writes global keys (vox_base + index, or the
//                 invalid key).
// The run list of the order follows: a run is the cells of one voxel, and
// each instance's non-secreting cells form one run marked kRunNone.
#include "pcg_kernels.cuh"

#include <algorithm>
#include <vector>

namespace pcg {

namespace {
constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr uint32_t kTile = kThreads * kItems;   // 2048 cells per tile
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kInvalid = 0xFFFFFFFFu;      // local key of a non-secreting cell
constexpr int kMaxDigitBits = 8;
constexpr uint32_t kMaxBins = (1u << kMaxDigitBits) + 1;   // digits + the non-secreting bin
}  // namespace

__device__ __forceinline__ uint32_t so_digit(uint32_t key, int shift, uint32_t R)
{
    return key == kInvalid ? R : (key >> shift) & (R - 1u);
}

// Digit counts of one tile; the first pass computes each cell's local key
// (its voxel index, or kInvalid) from the SoA and stores it in cell order.
template <bool FIRST>
__global__ void __launch_bounds__(kThreads) k_so_hist(const SegTile* __restrict__ tiles, const float* __restrict__ soa,
                                                      uint32_t stride, const CellInst* __restrict__ insts,
                                                      const uint8_t* __restrict__ active, uint32_t* __restrict__ keys,
                                                      int shift, uint32_t R, uint32_t* __restrict__ hist)
{
    __shared__ uint32_t cnt[kMaxBins];
    const SegTile tl = tiles[blockIdx.x];
    for (uint32_t d = threadIdx.x; d <= R; d += kThreads) cnt[d] = 0;
    __syncthreads();
    const CellInst& in = insts[tl.inst];
    const uint32_t nv = in.nx * in.ny * in.nz;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint32_t t = k * kThreads + threadIdx.x;
        if (t >= tl.count) continue;
        const uint32_t i = tl.first + t;
        uint32_t key;
        if (FIRST) {
            const uint32_t v = __float_as_uint(soa[static_cast<size_t>(F_VOXEL_IDX) * stride + i]);
            const bool ok = (active == nullptr || active[i] != 0) && v < nv && in.S > 0;
            key = ok ? v : kInvalid;
            keys[i] = key;
        } else {
            key = keys[i];
        }
        atomicAdd(&cnt[so_digit(key, shift, R)], 1u);
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d <= R; d += kThreads) hist[static_cast<size_t>(R + 1) * blockIdx.x + d] = cnt[d];
}

// Exclusive scan of one instance's counts in (digit, tile) order, in place:
// hist row t (R + 1 counts of tile t) becomes the first place of each of
// the tile's digit runs.  One block per instance with cells (inst_tile[b]
// = its first tile); thread j covers digits j, j + 256, ...  The rows of an
// instance's tiles are contiguous, so they come into shared memory (up to
// kOffSmem bytes of rows at a time) with coalesced loads, all in flight
// together, and go back the same way; the walks over tiles then read
// shared memory.
constexpr int kOffThreads = 256;
constexpr uint32_t kOffSmem = 46 * 1024;
__global__ void __launch_bounds__(kOffThreads, 1) k_so_offsets(const SegTile* __restrict__ tiles,
                                                            const uint32_t* __restrict__ inst_tile,
                                                            const CellInst* __restrict__ insts, uint32_t R,
                                                            uint32_t* __restrict__ hist)
{
    __shared__ uint32_t wsum[kOffThreads / 32];
    __shared__ uint32_t rows[kOffSmem / 4];
    const SegTile t0 = tiles[inst_tile[blockIdx.x]];
    const uint32_t nb = R + 1;
    const uint32_t chunk = (kOffSmem / 4) / nb;   // tiles per chunk (>= 44: nb <= 257)
    const bool one = t0.nt <= chunk;               // every row stays in shared memory
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr uint32_t kPer = (kMaxBins + kOffThreads - 1) / kOffThreads;   // digits per thread
    uint32_t tot[kPer];
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) tot[k] = 0;
    uint32_t* base = hist + static_cast<size_t>(nb) * t0.tb;
    for (uint32_t c0 = 0; c0 < t0.nt; c0 += chunk) {
        const uint32_t words = min(chunk, t0.nt - c0) * nb;
        const uint32_t* src = base + static_cast<size_t>(c0) * nb;
        for (uint32_t i = threadIdx.x; i < words; i += kOffThreads) rows[i] = src[i];
        __syncthreads();
        const uint32_t cn = words / nb;
#pragma unroll
        for (uint32_t k = 0; k < kPer; ++k) {
            const uint32_t d = threadIdx.x + k * kOffThreads;
            if (d < nb)
                for (uint32_t t = 0; t < cn; ++t) tot[k] += rows[t * nb + d];
        }
        __syncthreads();
    }
    // digits in order: digit d = threadIdx.x + k * 256, so the scan runs
    // over k-major blocks of 256 digits; start[k]: the first place of
    // this thread's digit k
    uint32_t run = insts[t0.inst].cell_off;
    uint32_t first[kPer];
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
        uint32_t incl = tot[k];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t before = 0, all = 0;
        for (int w = 0; w < kOffThreads / 32; ++w) {
            const uint32_t x = wsum[w];
            before += w < warp ? x : 0u;
            all += x;
        }
        __syncthreads();
        first[k] = run + before + incl - tot[k];
        run += all;
    }
    // each tile's row: the running place of every digit, tiles in order
    for (uint32_t c0 = 0; c0 < t0.nt; c0 += chunk) {
        const uint32_t words = min(chunk, t0.nt - c0) * nb;
        uint32_t* dst = base + static_cast<size_t>(c0) * nb;
        if (!one) {
            for (uint32_t i = threadIdx.x; i < words; i += kOffThreads) rows[i] = dst[i];
            __syncthreads();
        }
        const uint32_t cn = words / nb;
#pragma unroll
        for (uint32_t k = 0; k < kPer; ++k) {
            const uint32_t d = threadIdx.x + k * kOffThreads;
            if (d < nb) {
                uint32_t at = first[k];
                for (uint32_t t = 0; t < cn; ++t) {
                    const uint32_t c = rows[t * nb + d];
                    rows[t * nb + d] = at;
                    at += c;
                }
                first[k] = at;
            }
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < words; i += kOffThreads) dst[i] = rows[i];
        __syncthreads();
    }
}

template <bool FIRST, bool LAST>
__global__ void __launch_bounds__(kThreads) k_so_scatter(const SegTile* __restrict__ tiles,
                                                         const uint32_t* __restrict__ kin,
                                                         const uint32_t* __restrict__ vin,
                                                         uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                         int shift, uint32_t R, const uint32_t* __restrict__ offs,
                                                         const CellInst* __restrict__ insts, uint32_t invalid_key,
                                                         const double* __restrict__ cc, double* __restrict__ cs,
                                                         uint32_t cap, const uint32_t* __restrict__ flags)
{
    __shared__ uint32_t wcnt[kWarps][kMaxBins];
    __shared__ uint32_t cnt[kMaxBins];
    __shared__ uint32_t tbase[kMaxBins];
    __shared__ uint32_t gbase[kMaxBins];
    __shared__ uint32_t sk[kTile], sv[kTile];
    __shared__ uint32_t wsum[kWarps + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const SegTile tl = tiles[blockIdx.x];
    for (uint32_t d = threadIdx.x; d <= R; d += kThreads) {
#pragma unroll
        for (int w = 0; w < kWarps; ++w) wcnt[w][d] = 0;
        gbase[d] = offs[static_cast<size_t>(R + 1) * blockIdx.x + d];
    }
    uint32_t kk[kItems], vv[kItems], rk[kItems], dg[kItems];
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
        const uint32_t t = warp * (32 * kItems) + r * 32 + lane;
        const bool ok = t < tl.count;
        const uint32_t i = tl.first + t;
        kk[r] = ok ? kin[i] : 0u;
        vv[r] = ok ? (FIRST ? i : vin[i]) : 0u;
        dg[r] = ok ? so_digit(kk[r], shift, R) : R + 1u;   // R + 1 marks an empty lane
    }
    __syncthreads();
    // stable ranks within each warp's 256 keys, against the warp's own counts
    const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
        const uint32_t peers = __match_any_sync(0xffffffffu, dg[r]);
        const bool ok = dg[r] <= R;
        rk[r] = (ok ? wcnt[warp][dg[r]] : 0u) + __popc(peers & lt_mask);
        __syncwarp();
        if (ok && lane == __ffs(peers) - 1) wcnt[warp][dg[r]] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // warps in order: each warp's counts become its first place within the digit
    for (uint32_t d = threadIdx.x; d <= R; d += kThreads) {
        uint32_t sum = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = wcnt[w][d];
            wcnt[w][d] = sum;
            sum += c;
        }
        cnt[d] = sum;
    }
    __syncthreads();
    // exclusive scan of the tile's digit counts: thread t covers a run of
    // consecutive digits
    {
        const uint32_t per = (R + 1u + kThreads - 1u) / kThreads;
        const uint32_t d0 = threadIdx.x * per;
        uint32_t sum = 0;
        for (uint32_t d = d0; d < d0 + per && d <= R; ++d) sum += cnt[d];
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t before = 0;
        for (int w = 0; w < warp; ++w) before += wsum[w];
        uint32_t run = before + incl - sum;
        for (uint32_t d = d0; d < d0 + per && d <= R; ++d) {
            tbase[d] = run;
            run += cnt[d];
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
        if (dg[r] <= R) {
            const uint32_t t = tbase[dg[r]] + wcnt[warp][dg[r]] + rk[r];
            sk[t] = kk[r];
            sv[t] = vv[r];
        }
    }
    __syncthreads();
    const CellInst& in = insts[tl.inst];
    const uint32_t vox_base = LAST ? in.vox_base : 0u;
    // the last pass also moves the secretion constants of every secreting
    // cell (cc, in cell order) to its place in the order (cs): rate slot
    // rate_off + (place - cell_off) * S; c0 / c1 only where the instance
    // has them (flags)
    const bool consts = LAST && cc != nullptr;
    const uint32_t S = in.S, f = consts ? flags[tl.inst] : 0u;
    for (uint32_t t = threadIdx.x; t < tl.count; t += kThreads) {
        const uint32_t k = sk[t];
        const uint32_t d = so_digit(k, shift, R);
        const uint32_t dst = gbase[d] + (t - tbase[d]);
        const uint32_t g = sv[t];
        kout[dst] = LAST ? (k == kInvalid ? invalid_key : vox_base + k) : k;
        vout[dst] = g;
        if (consts && k != kInvalid) {
            const uint64_t src = in.rate_off + static_cast<uint64_t>(g - in.cell_off) * S;
            const uint64_t to = in.rate_off + static_cast<uint64_t>(dst - in.cell_off) * S;
            if (S == 2 && f == 0) {   // the common uptake-only case: c2 of both substrates
                const double a = cc[2ull * cap + src], b = cc[2ull * cap + src + 1];
                cs[2ull * cap + to] = a;
                cs[2ull * cap + to + 1] = b;
            } else {
                for (uint32_t q = 0; q < S; ++q) {
                    if (f & 1u) cs[to + q] = cc[src + q];
                    if (f & 2u) cs[cap + to + q] = cc[cap + src + q];
                    cs[2ull * cap + to + q] = cc[2ull * cap + src + q];
                }
            }
        }
    }
}

// Runs of the order: a run starts where the key changes (each instance's
// non-secreting cells, key invalid_key, form one run).  Positions go in
// tiles of 2048, position base + k * 256 + t to thread t (k = 0..7), so
// every warp access is contiguous: k_so_run_count counts each tile's run
// heads, their exclusive scan gives each tile its first run index, and
// k_so_run_write numbers the tile's heads (ballots, then the 64 warp-row
// counts in order) and writes the runs.  Run r starts at run_start[r] and
// ends at run_start[r + 1] (run_start[n_runs] = n, *n_runs = the count).
// A run of secreting cells gets one word: its instance and the density
// element of its voxel (substrate 0, padded rows); a run of non-secreting
// cells gets kRunNone.
__device__ __forceinline__ bool so_head(const uint32_t* __restrict__ skeys, uint32_t n, uint32_t p, uint32_t* key)
{
    if (p >= n) return false;
    *key = skeys[p];
    return p == 0 || skeys[p - 1] != *key;
}

__global__ void __launch_bounds__(kThreads) k_so_run_count(const uint32_t* __restrict__ skeys, uint32_t n,
                                                           uint32_t* __restrict__ tile_cnt)
{
    __shared__ uint32_t ws[kWarps];
    uint32_t c = 0, key;
#pragma unroll
    for (int k = 0; k < kItems; ++k) c += so_head(skeys, n, blockIdx.x * kTile + k * kThreads + threadIdx.x, &key);
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) t += ws[w];
        tile_cnt[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kThreads) k_so_run_write(const uint32_t* __restrict__ skeys,
                                                           const uint32_t* __restrict__ sorder, uint32_t n,
                                                           uint32_t invalid_key, const uint32_t* __restrict__ tile_off,
                                                           const uint32_t* __restrict__ tile_cnt, uint32_t ntiles,
                                                           const uint32_t* __restrict__ cell_inst,
                                                           const CellInst* __restrict__ insts,
                                                           uint32_t* __restrict__ run_start,
                                                           uint64_t* __restrict__ run_word, uint32_t* __restrict__ n_runs)
{
    __shared__ uint32_t wc[kItems * kWarps];   // heads per (row k, warp), then their exclusive scan
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t key[kItems], hb = 0, rank[kItems];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const bool h = so_head(skeys, n, blockIdx.x * kTile + k * kThreads + threadIdx.x, &key[k]);
        const uint32_t b = __ballot_sync(0xffffffffu, h);
        hb |= (h ? 1u : 0u) << k;
        rank[k] = __popc(b & lt_mask);
        if (lane == 0) wc[k * kWarps + warp] = __popc(b);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = tile_off[blockIdx.x];
        for (int i = 0; i < kItems * kWarps; ++i) {
            const uint32_t c = wc[i];
            wc[i] = run;
            run += c;
        }
    }
    __syncthreads();
    uint32_t ii8[kItems];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const bool sec = ((hb >> k) & 1u) && key[k] < invalid_key;
        ii8[k] = sec ? sorder[blockIdx.x * kTile + k * kThreads + threadIdx.x] : 0u;
    }
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const bool sec = ((hb >> k) & 1u) && key[k] < invalid_key;
        ii8[k] = sec ? cell_inst[ii8[k]] : kRunNone;
    }
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        if (!((hb >> k) & 1u)) continue;
        const uint32_t p = blockIdx.x * kTile + k * kThreads + threadIdx.x;
        const uint32_t r = wc[k * kWarps + warp] + rank[k];
        const uint32_t ii = ii8[k];
        run_start[r] = p;
        uint64_t elem = 0;
        if (ii != kRunNone) {
            const CellInst& in = insts[ii];
            const uint32_t v = key[k] - in.vox_base;
            elem = in.dens_off + static_cast<uint64_t>(v / in.nx) * in.px + v % in.nx;
        }
        run_word[r] = make_run_word(ii, elem);
    }
    if (blockIdx.x == ntiles - 1 && threadIdx.x == 0) {
        const uint32_t total = tile_off[blockIdx.x] + tile_cnt[blockIdx.x];
        run_start[total] = n;
        *n_runs = total;
    }
}

// ------------------------------------------------------------------ host

void so_plan(uint32_t max_local_voxels, int* passes, int* digit_bits)
{
    int bits = 0;
    while ((1ull << bits) < max_local_voxels) ++bits;
    const int p = bits == 0 ? 1 : (bits + kMaxDigitBits - 1) / kMaxDigitBits;
    *passes = p;
    *digit_bits = (bits + p - 1) / p;
}

uint32_t so_max_tiles(uint32_t max_cells, uint32_t n_inst) { return max_cells / kTile + n_inst + 1; }

void so_tiles(const CellInst* inst, uint32_t n_inst, std::vector<SegTile>& out, std::vector<uint32_t>& inst_tile)
{
    out.clear();
    inst_tile.clear();
    for (uint32_t i = 0; i < n_inst; ++i) {
        const uint32_t nt = (inst[i].n_cells + kTile - 1) / kTile;
        const uint32_t tb = static_cast<uint32_t>(out.size());
        if (nt) inst_tile.push_back(tb);
        for (uint32_t t = 0; t < nt; ++t) {
            SegTile s{};
            s.first = inst[i].cell_off + t * kTile;
            s.count = std::min(kTile, inst[i].n_cells - t * kTile);
            s.inst = i;
            s.tb = tb;
            s.nt = nt;
            out.push_back(s);
        }
    }
}

size_t so_scratch_bytes(uint32_t max_tiles)
{
    return static_cast<size_t>(max_tiles) * kMaxBins * sizeof(uint32_t);
}

static uint32_t run_tiles(uint32_t n) { return (n + kTile - 1) / kTile; }

size_t so_run_scratch_bytes(uint32_t max_cells)
{
    const uint64_t rt = run_tiles(max_cells) + 1;
    return 2 * ((rt * sizeof(uint32_t) + 255) / 256) * 256 + scan_scratch_bytes(rt);
}

int so_launches(uint32_t ntiles, int passes, uint32_t n)
{
    if (n == 0 || ntiles == 0) return 0;
    return passes * 3 + 2 + scan_launches(run_tiles(n));
}

cudaError_t launch_sec_order(cudaStream_t st, const SegTile* tiles, uint32_t ntiles, const uint32_t* inst_tile,
                             uint32_t n_inst_tiled, uint32_t n, int passes,
                             int digit_bits, const float* soa, uint32_t stride, const CellInst* insts,
                             const uint8_t* active, const uint32_t* cell_inst, uint32_t invalid_key, uint32_t* keys,
                             uint32_t* ktmp, uint32_t* vtmp, uint32_t* skeys, uint32_t* sorder, void* scratch,
                             uint32_t* n_runs, uint32_t* run_start, uint64_t* run_word, void* run_scratch,
                             const double* cc, double* cs, uint32_t cap, const uint32_t* flags)
{
    if (n == 0 || ntiles == 0) return cudaSuccess;
    if (digit_bits > kMaxDigitBits || passes < 1) return cudaErrorInvalidValue;
    const uint32_t R = 1u << digit_bits;
    uint32_t* hist = static_cast<uint32_t*>(scratch);
    const uint32_t* ks = keys;
    const uint32_t* vs = nullptr;
    cudaError_t e;
    for (int p = 0; p < passes; ++p) {
        const bool first = p == 0, last = p == passes - 1;
        // the last pass writes (skeys, sorder); earlier ones alternate so that it does
        const bool to_out = ((passes - 1 - p) & 1) == 0;
        uint32_t* kd = to_out ? skeys : ktmp;
        uint32_t* vd = to_out ? sorder : vtmp;
        const int shift = p * digit_bits;
        if (first)
            k_so_hist<true><<<ntiles, kThreads, 0, st>>>(tiles, soa, stride, insts, active, keys, shift, R, hist);
        else
            k_so_hist<false><<<ntiles, kThreads, 0, st>>>(tiles, soa, stride, insts, active, const_cast<uint32_t*>(ks),
                                                           shift, R, hist);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        k_so_offsets<<<n_inst_tiled, kOffThreads, 0, st>>>(tiles, inst_tile, insts, R, hist);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
#define PCG_SO_SCATTER(F, L)                                                                                    \
    k_so_scatter<F, L><<<ntiles, kThreads, 0, st>>>(tiles, ks, vs, kd, vd, shift, R, hist, insts, invalid_key, cc, cs, \
                                                    cap, flags)
        if (first && last) PCG_SO_SCATTER(true, true);
        else if (first) PCG_SO_SCATTER(true, false);
        else if (last) PCG_SO_SCATTER(false, true);
        else PCG_SO_SCATTER(false, false);
#undef PCG_SO_SCATTER
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        ks = kd;
        vs = vd;
    }
    const uint32_t rt = run_tiles(n);
    uint32_t* tile_cnt = static_cast<uint32_t*>(run_scratch);
    uint32_t* tile_off = tile_cnt + ((static_cast<uint64_t>(rt + 1) * sizeof(uint32_t) + 255) / 256) * 256 / sizeof(uint32_t);
    char* rscr = reinterpret_cast<char*>(tile_off) + ((static_cast<uint64_t>(rt + 1) * sizeof(uint32_t) + 255) / 256) * 256;
    k_so_run_count<<<rt, kThreads, 0, st>>>(skeys, n, tile_cnt);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = scan_exclusive(st, tile_cnt, tile_off, rt, rscr)) != cudaSuccess) return e;
    k_so_run_write<<<rt, kThreads, 0, st>>>(skeys, sorder, n, invalid_key, tile_off, tile_cnt, rt, cell_inst, insts,
                                             run_start, run_word, n_runs);
    return cudaGetLastError();
}

}  // namespace pcg
