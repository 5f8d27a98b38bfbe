// sort.cu — stable LSD radix sort of (key, value) pairs and a warp-shuffle
// exclusive scan (sm_100a).  The sort backs pcg_sort_pairs_static (the
// secretion order has its own instance-segmented sort, secorder.cu); the
// scan turns the per-voxel counts of the mechanics binning into the
// cell-start table, and serves the sort's digit histograms and the
// secretion run list's tile counts.
//
// One radix pass over D-bit digits:
//   k_radix_hist     per-tile digit histogram -> hist[digit * tiles + tile]
//   scan_exclusive   over hist (digit-major, so equal digits keep tile order)
//   k_radix_scatter  each warp ranks its contiguous 256 keys with
//                    __match_any_sync (peers with the same digit) and a
//                    per-warp running count, warps are combined in warp
//                    order; the tile is laid out in shared memory in digit
//                    order and written back so that consecutive threads
//                    store consecutive elements of one digit's run at
//                    offset[digit][tile] + place in the run.
// Ranks follow input order within a warp, warps follow tile order and
// tiles follow the scanned histogram, so each pass is stable.
#include "pcg_kernels.cuh"

namespace pcg {

namespace {
constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;     // 2048 keys per tile
constexpr int kWarps = kThreads / 32;
constexpr int kDigitBits = 8;
constexpr int kRadix = 1 << kDigitBits;
constexpr uint32_t kMask = kRadix - 1;
}  // namespace

__global__ void __launch_bounds__(kThreads) k_radix_hist(const uint32_t* __restrict__ keys, uint32_t n, int shift,
                                                         uint32_t* __restrict__ hist, uint32_t ntiles)
{
    __shared__ uint32_t h[kRadix];
    for (int i = threadIdx.x; i < kRadix; i += kThreads) h[i] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * kTile;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint32_t i = base + k * kThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & kMask], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kThreads) hist[d * ntiles + blockIdx.x] = h[d];
}

__global__ void __launch_bounds__(kThreads) k_radix_scatter(const uint32_t* __restrict__ kin,
                                                            const uint32_t* __restrict__ vin,
                                                            uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                            uint32_t n, int shift,
                                                            const uint32_t* __restrict__ offsets, uint32_t ntiles)
{
    __shared__ uint32_t wcnt[kWarps][kRadix];
    __shared__ uint32_t gbase[kRadix];
    __shared__ uint32_t tbase[kRadix];      // first place of each digit in the tile
    __shared__ uint32_t wtot[kWarps];
    __shared__ uint32_t sk[kTile], sv[kTile];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kThreads) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t base = blockIdx.x * kTile + warp * (32 * kItems);
    uint32_t kk[kItems], vv[kItems], rk[kItems];
    int dg[kItems];
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
        const uint32_t i = base + r * 32 + lane;
        const bool ok = i < n;
        kk[r] = ok ? kin[i] : 0u;
        vv[r] = ok ? vin[i] : 0u;
        dg[r] = ok ? static_cast<int>((kk[r] >> shift) & kMask) : kRadix;   // kRadix marks an empty lane
        const uint32_t peers = __match_any_sync(0xffffffffu, dg[r]);
        rk[r] = (ok ? wcnt[warp][dg[r]] : 0u) + __popc(peers & lt);
        __syncwarp();
        if (ok && lane == __ffs(peers) - 1) wcnt[warp][dg[r]] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    static_assert(kThreads == kRadix, "one thread per digit");
    {
        const int d = threadIdx.x;
        uint32_t sum = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = wcnt[w][d];
            wcnt[w][d] = sum;
            sum += c;
        }
        gbase[d] = offsets[d * ntiles + blockIdx.x];
        // exclusive scan of the digit totals across the block
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wtot[warp] = incl;
        __syncthreads();
        uint32_t before = 0;
        for (int w = 0; w < warp; ++w) before += wtot[w];
        tbase[d] = before + incl - sum;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
        if (dg[r] < kRadix) {
            const uint32_t t = tbase[dg[r]] + wcnt[warp][dg[r]] + rk[r];
            sk[t] = kk[r];
            sv[t] = vv[r];
        }
    }
    __syncthreads();
    const uint32_t count = min(static_cast<uint32_t>(kTile), n - blockIdx.x * kTile);
    for (uint32_t t = threadIdx.x; t < count; t += kThreads) {
        const uint32_t k = sk[t];
        const int d = static_cast<int>((k >> shift) & kMask);
        const uint32_t dst = gbase[d] + (t - tbase[d]);
        kout[dst] = k;
        vout[dst] = sv[t];
    }
}

// ------------------------------------------------------------------ scan

// Scans over more than one tile reduce, then scan: k_tile_sums writes every
// tile's total, the totals are scanned (recursively), and k_scan_tiles
// scans every tile once more, starting from its scanned total -- one read
// pass and one read / write pass over the values.

// Sum of one 2048-value tile per block.
__global__ void __launch_bounds__(kThreads) k_tile_sums(const uint32_t* __restrict__ in, uint64_t n,
                                                        uint32_t* __restrict__ sums)
{
    __shared__ uint32_t wsum[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kTile + static_cast<uint64_t>(threadIdx.x) * kItems;
    uint32_t tot = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint64_t i = base + k;
        tot += i < n ? in[i] : 0u;
    }
    tot = __reduce_add_sync(0xffffffffu, tot);
    if (lane == 0) wsum[warp] = tot;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) t += wsum[w];
        sums[blockIdx.x] = t;
    }
}

// Exclusive scan of 256 per-thread values across the block: returns the
// sum of the values of the threads before this one; *total gets the sum of
// all (wsum: kWarps + 1 shared words).
__device__ __forceinline__ uint32_t block_exclusive(uint32_t x, uint32_t* wsum, uint32_t* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < kWarps ? wsum[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < kWarps; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < kWarps) wsum[lane] = wi - w;
        if (lane == kWarps - 1) wsum[kWarps] = wi;
    }
    __syncthreads();
    const uint32_t before = wsum[warp] + (incl - x);
    *total = wsum[kWarps];
    __syncthreads();   // wsum is reused by the next call
    return before;
}

// Exclusive scan of one 2048-value tile per block, each tile starting from
// offs[blockIdx.x] when offs != nullptr.  The tile is two halves of 1024
// values; in each, thread t owns values 4t .. 4t + 3, moved as one 16-byte
// access when the tile is whole and the arrays 16-byte aligned, so that a
// warp's loads and stores are contiguous.
__global__ void __launch_bounds__(kThreads) k_scan_tiles(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                         uint64_t n, const uint32_t* __restrict__ offs)
{
    static_assert(kTile == 2 * 4 * kThreads, "two halves of four values per thread");
    __shared__ uint32_t wsum[kWarps + 1];
    const uint64_t tile = static_cast<uint64_t>(blockIdx.x) * kTile;
    const bool vec = tile + kTile <= n && ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u) == 0;
    uint32_t run = offs ? offs[blockIdx.x] : 0u;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const uint64_t i0 = tile + static_cast<uint64_t>(h) * (kTile / 2) + 4ull * threadIdx.x;
        uint32_t v[4];
        if (vec) {
            const uint4 q = *reinterpret_cast<const uint4*>(in + i0);
            v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) v[k] = i0 + k < n ? in[i0 + k] : 0u;
        }
        uint32_t tot = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t x = v[k];
            v[k] = tot;
            tot += x;
        }
        uint32_t half_total = 0;
        const uint32_t pre = run + block_exclusive(tot, wsum, &half_total);
        if (vec) {
            *reinterpret_cast<uint4*>(out + i0) = make_uint4(v[0] + pre, v[1] + pre, v[2] + pre, v[3] + pre);
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (i0 + k < n) out[i0 + k] = v[k] + pre;
        }
        run += half_total;
    }
}

static uint64_t tiles_of(uint64_t n) { return (n + kTile - 1) / kTile; }

cudaError_t sort_kernels_load()
{
    // querying a kernel's attributes loads its module on the current device
    // (lazy loading defers that to the first launch otherwise)
    cudaFuncAttributes a;
    const void* ks[] = {reinterpret_cast<const void*>(&k_radix_hist), reinterpret_cast<const void*>(&k_radix_scatter),
                        reinterpret_cast<const void*>(&k_scan_tiles), reinterpret_cast<const void*>(&k_tile_sums)};
    for (const void* k : ks) {
        const cudaError_t e = cudaFuncGetAttributes(&a, k);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

size_t scan_scratch_bytes(uint64_t n)
{
    size_t bytes = 0;
    uint64_t m = tiles_of(n);
    while (m > 1) {
        bytes += ((m * sizeof(uint32_t) + 255) / 256) * 256;
        m = tiles_of(m);
    }
    return bytes + 256;
}

int scan_launches(uint64_t n)
{
    const uint64_t nt = tiles_of(n);
    return nt <= 1 ? 1 : 2 + scan_launches(nt);
}

static cudaError_t scan_rec(cudaStream_t st, const uint32_t* in, uint32_t* out, uint64_t n, char* scratch)
{
    const uint64_t nt = tiles_of(n);
    if (nt == 0) return cudaSuccess;
    if (nt == 1) {
        k_scan_tiles<<<1, kThreads, 0, st>>>(in, out, n, nullptr);
        return cudaGetLastError();
    }
    uint32_t* sums = reinterpret_cast<uint32_t*>(scratch);
    char* next = scratch + ((nt * sizeof(uint32_t) + 255) / 256) * 256;
    k_tile_sums<<<static_cast<unsigned>(nt), kThreads, 0, st>>>(in, n, sums);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = scan_rec(st, sums, sums, nt, next);
    if (e != cudaSuccess) return e;
    k_scan_tiles<<<static_cast<unsigned>(nt), kThreads, 0, st>>>(in, out, n, sums);
    return cudaGetLastError();
}

cudaError_t scan_exclusive(cudaStream_t st, const uint32_t* in, uint32_t* out, uint64_t n, void* scratch)
{
    return scan_rec(st, in, out, n, static_cast<char*>(scratch));
}

// ------------------------------------------------------------------ sort

static int passes_for(int bits) { return bits <= 0 ? 0 : (bits + kDigitBits - 1) / kDigitBits; }

size_t radix_sort_scratch_bytes(uint32_t n, int bits)
{
    (void)bits;
    const uint64_t nt = tiles_of(n ? n : 1);
    const uint64_t hist = nt * kRadix;
    return ((hist * sizeof(uint32_t) + 255) / 256) * 256 + scan_scratch_bytes(hist);
}

int radix_sort_launches(uint32_t n, int bits)
{
    const uint64_t nt = tiles_of(n ? n : 1);
    const int p = passes_for(bits);
    if (p == 0) return 2;
    return p * (2 + scan_launches(nt * kRadix));
}

cudaError_t radix_sort_pairs(cudaStream_t st, const uint32_t* k_in, const uint32_t* v_in, uint32_t* k_out,
                             uint32_t* v_out, uint32_t* k_tmp, uint32_t* v_tmp, uint32_t n, int bits, void* scratch)
{
    if (n == 0) return cudaSuccess;
    const uint32_t nt = static_cast<uint32_t>(tiles_of(n));
    uint32_t* hist = static_cast<uint32_t*>(scratch);
    char* sscr = static_cast<char*>(scratch) + ((static_cast<uint64_t>(nt) * kRadix * sizeof(uint32_t) + 255) / 256) * 256;
    const int passes = passes_for(bits);
    if (passes == 0) {
        cudaError_t e = cudaMemcpyAsync(k_out, k_in, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return e;
        return cudaMemcpyAsync(v_out, v_in, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    }
    // ping-pong so that the last pass writes (k_out, v_out)
    const uint32_t* ks = k_in;
    const uint32_t* vs = v_in;
    for (int p = 0; p < passes; ++p) {
        const bool last = p == passes - 1;
        // pass p writes out when (passes - 1 - p) is even, tmp otherwise
        const bool to_out = ((passes - 1 - p) & 1) == 0;
        uint32_t* kd = to_out ? k_out : k_tmp;
        uint32_t* vd = to_out ? v_out : v_tmp;
        const int shift = p * kDigitBits;
        k_radix_hist<<<nt, kThreads, 0, st>>>(ks, n, shift, hist, nt);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        e = scan_exclusive(st, hist, hist, static_cast<uint64_t>(nt) * kRadix, sscr);
        if (e != cudaSuccess) return e;
        k_radix_scatter<<<nt, kThreads, 0, st>>>(ks, vs, kd, vd, n, shift, hist, nt);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        ks = kd;
        vs = vd;
        (void)last;
    }
    return cudaSuccess;
}

}  // namespace pcg
