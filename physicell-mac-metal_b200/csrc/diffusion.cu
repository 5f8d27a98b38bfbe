// diffusion.cu — LOD Thomas sweeps, Dirichlet reset and gradients (sm_100a).
//
// Reference semantics: shaders/diffusion_2d.metal:28-157 (x sweep) and
// :165-292 (y sweep), one tridiagonal solve per line over the interior
// nodes 1..n-2 with the decay on the diagonal; src/microenvironment.mm:127-152
// (applyDirichletBC); :282-342 (computeGradients).  The z sweep applies the
// same per-line rule along k.
//
// The solve.  Every line of one (instance, substrate, axis) family has the
// same matrix, so g_i = c / den_i and 1 / den_i are one table (LineRule,
// built in FP64 on the host).  With h_i = (rho_i + fold_i) / den_i the
// reference's two passes are
//     forward   d_i = g_i d_{i-1} + h_i        (d_0 = 0)
//     backward  x_i = g_i x_{i+1} + d_i        (x_{n-1} = 0)
// one FMUL + one FFMA, then one FFMA per value.  End nodes keep their value
// or take the Dirichlet target.
//
// Data movement.  density is [s][k][j][i] FP32 with rows padded to a pitch
// px = nx rounded up to 4 floats, so every row starts on 16 bytes.  Each
// warp of a persistent CTA runs its own pipeline of shared-memory stages:
// lane 0 issues one TMA tensor copy (cp.async.bulk.tensor) of the warp's
// next tile into a free stage, completion is counted on one mbarrier per
// stage, the warp solves the current stage in place and writes it back with
// one tensor store.  Tiles are loaded while the previous one is solved, so
// HBM sees a deep queue with few threads.
//   x tile:   32 lines (one per lane) stored [line][P], P = row_smem_pitch(nx)
//             (2-D map, box P x 32); all lanes walk their lines in step,
//             4 values per 16-byte shared access, coefficients broadcast;
//   y/z tile: 32 adjacent columns x n rows stored [row][32] (3-D map, box
//             32 x n); lane = column.
// Lines too long for a tensor box move with 1-D bulk copies (x: the whole
// tile, lanes skewed by the lane index so 32 lanes hit 32 banks; y/z: one
// 128-byte copy per row).
// Every value is read from HBM once and written once per sweep.  Waits are
// bounded: a wait that runs out records PCG_DEV_TIMEOUT in the status word,
// drains what it issued, and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "pcg_kernels.cuh"

namespace pcg {

// The LineRule a tile descriptor carries.
__device__ __forceinline__ LineRule rule_of(const SweepTile& t)
{
    LineRule r;
    r.tab = t.tab;
    r.n = t.n;
    r.c = 0.f;
    r.fold = t.fold;
    r.T = t.T;
    r.dir = t.inst >> 31;
    r.inst = t.inst & 0x7fffffffu;
    r._pad = 0;
    return r;
}

__device__ __forceinline__ bool tile_on(const LineRule& r, const uint8_t* __restrict__ mask)
{
    return mask == nullptr || (mask[r.inst] & STEP_DIFFUSE);
}

// Column tile lane -> (slab, column).
__device__ __forceinline__ uint32_t lane_slab(const SweepTile& tile, int lane) { return static_cast<uint32_t>(lane) / tile.width; }
__device__ __forceinline__ uint32_t lane_col(const SweepTile& tile, int lane) { return static_cast<uint32_t>(lane) % tile.width; }

// The lane's line lies on a face of the block (3-D: x faces and, for z
// lines, y faces; 2-D y lines: x faces).
__device__ __forceinline__ bool on_face(const SweepTile& tile, int lane)
{
    const uint32_t i = tile.i0 + lane_col(tile, lane);
    if (i == 0u || i + 1u == tile.nx) return true;
    if (tile.face & TILE_AXIS_Z) {
        const uint32_t j = tile.outer + lane_slab(tile, lane);
        return j == 0u || j + 1u == tile.outer_n;
    }
    return false;
}

// ------------------------------------------------------------------ TMA / mbarrier helpers

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// One bounded try: the thread may be suspended for up to kSuspendNs while
// the phase is incomplete, so a waiting warp does not spin on the issue
// slots of the warps that are computing.
constexpr uint32_t kSuspendNs = 20000;

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendNs)
        : "memory");
    return done != 0;
}

// Bounded wait: about one second of SM clock, then PCG_DEV_TIMEOUT.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned* status)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > (2ll << 30)) {
            atomicOr(status, PCG_DEV_TIMEOUT);
            return false;
        }
    }
    return true;
}

// global -> shared, completion counted on 'bar' (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gsrc, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(smem_dst)),
                 "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// shared -> global in this thread's bulk group
__device__ __forceinline__ void bulk_store(void* gdst, const void* smem_src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_u32(smem_src)),
                 "r"(bytes)
                 : "memory");
}
// 3-D tensor-map copies of a whole column tile (one instruction each way)
__device__ __forceinline__ void tensor_load3(void* smem_dst, const void* tmap, int c0, int c1, int c2, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
            "r"(smem_u32(smem_dst)),
        "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
// 2-D tensor-map copies of a whole x tile
__device__ __forceinline__ void tensor_load2(void* smem_dst, const void* tmap, int c0, int c1, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(smem_dst)),
        "l"(tmap), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}
// L2 prefetch of a tensor box (no shared memory, no barrier): the box a
// later CTA will load then comes from L2.
__device__ __forceinline__ void tensor_prefetch2(const void* tmap, int c0, int c1)
{
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(tmap), "r"(c0), "r"(c1)
                 : "memory");
}
__device__ __forceinline__ void tensor_prefetch3(const void* tmap, int c0, int c1, int c2)
{
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(tmap), "r"(c0), "r"(c1),
                 "r"(c2)
                 : "memory");
}
__device__ __forceinline__ void tensor_store2(const void* tmap, int c0, int c1, const void* smem_src)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(tmap), "r"(c0),
                 "r"(c1), "r"(smem_u32(smem_src))
                 : "memory");
}
__device__ __forceinline__ void tensor_store3(const void* tmap, int c0, int c1, int c2, const void* smem_src)
{
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(tmap),
                 "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(smem_src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ bool aligned16(const void* p, uint32_t bytes)
{
    return ((reinterpret_cast<uintptr_t>(p) | bytes) & 15u) == 0 && bytes > 0;
}

// ------------------------------------------------------------------ tile geometry

// Bytes of one row copy of a column tile (count columns rounded up to 4).
__device__ __forceinline__ uint32_t col_row_bytes(uint32_t count) { return ((count + 3u) & ~3u) * 4u; }

// Issue the loads of 'tile' into stage 'st' (all lanes take part).
// Tensor coordinates of a column tile's box: (x, slab, line position).
__device__ __forceinline__ void tile_coords(const SweepTile& tile, int* c)
{
    c[0] = static_cast<int>(tile.i0);
    c[1] = static_cast<int>(tile.outer);
    c[2] = 0;
}

// Issue the loads of 'tile' into stage 'st' and of its rule's coefficient
// table into 'stab' (the stage's table area), all counted on 'bar'.
template <bool kRows>
__device__ __forceinline__ bool issue_tile_load(const SweepTile& tile, const float* __restrict__ dens,
                                                const float* __restrict__ tab, const void* tmaps, float* st,
                                                float* stab, uint64_t* bar, int lane, unsigned* status)
{
    const LineRule r = rule_of(tile);
    const uint32_t n = r.n;
    const uint32_t tb = tab_floats(n) * 4u;    // 32-byte multiple, 32-byte aligned source
    const float* src = dens + tile.base;
    const void* map = static_cast<const unsigned char*>(tmaps) + static_cast<size_t>(tile.map) * 128;
    if (kRows && (tile.face & TILE_TENSOR)) {
        if (lane == 0) {
            mbar_arrive_expect_tx(bar, 32u * row_smem_pitch(n) * 4u + tb);   // the whole box, fill included
            tensor_load2(st, map, 0, static_cast<int>(tile.outer), bar);
            bulk_load(stab, tab + r.tab, tb, bar);
        }
        return true;
    }
    if (!kRows && (tile.face & TILE_TENSOR)) {
        if (lane == 0) {
            int c[3];
            tile_coords(tile, c);
            mbar_arrive_expect_tx(bar, 32u * n * 4u + tb);
            tensor_load3(st, map, c[0], c[1], c[2], bar);
            bulk_load(stab, tab + r.tab, tb, bar);
        }
        return true;
    }
    if (kRows) {
        const uint32_t bytes = tile.count * tile.rs * 4u;     // count lines of pitch rs
        if (lane == 0) {
            if (!aligned16(src, bytes)) {
                atomicOr(status, PCG_DEV_ALIGN);
                mbar_arrive_expect_tx(bar, 0);
                return false;
            }
            mbar_arrive_expect_tx(bar, bytes + tb);
            bulk_load(st, src, bytes, bar);
            bulk_load(stab, tab + r.tab, tb, bar);
        }
    } else {
        const uint32_t rb = col_row_bytes(tile.count);
        if (!aligned16(src, rb) || (tile.rs & 3u)) {
            if (lane == 0) {
                atomicOr(status, PCG_DEV_ALIGN);
                mbar_arrive_expect_tx(bar, 0);
            }
            return false;
        }
        if (lane == 0) {
            mbar_arrive_expect_tx(bar, rb * n + tb);
            bulk_load(stab, tab + r.tab, tb, bar);
        }
        __syncwarp();
        for (uint32_t j = lane; j < n; j += 32) bulk_load(st + j * 32, src + static_cast<size_t>(j) * tile.rs, rb, bar);
    }
    return true;
}

template <bool kRows>
__device__ __forceinline__ void issue_tile_store(const SweepTile& tile, float* __restrict__ dens, const void* tmaps, const float* st, int lane)
{
    float* dst = dens + tile.base;
    if (kRows && (tile.face & TILE_TENSOR)) {
        if (lane == 0) {
            tensor_store2(static_cast<const unsigned char*>(tmaps) + static_cast<size_t>(tile.map) * 128, 0,
                          static_cast<int>(tile.outer), st);
            bulk_commit();
        }
        return;
    }
    if (!kRows && (tile.face & TILE_TENSOR)) {
        if (lane == 0) {
            int c[3];
            tile_coords(tile, c);
            tensor_store3(static_cast<const unsigned char*>(tmaps) + static_cast<size_t>(tile.map) * 128, c[0], c[1],
                          c[2], st);
            bulk_commit();
        }
        return;
    }
    if (kRows) {
        if (lane == 0) {
            bulk_store(dst, st, tile.count * tile.rs * 4u);
            bulk_commit();
        }
    } else {
        const uint32_t n = tile.n;
        const uint32_t rb = col_row_bytes(tile.count);
        for (uint32_t j = lane; j < n; j += 32) bulk_store(dst + static_cast<size_t>(j) * tile.rs, st + j * 32, rb);
        bulk_commit();
    }
}

// ------------------------------------------------------------------ solves in shared memory

// Coefficient table of one rule: line positions in chunks of 4, each chunk
// 8 floats {g[4], inv[4]} (32-byte aligned), g_i = c / den_i, inv_i = 1 / den_i;
// zero at the end nodes.  The tile solves read the copy staged in shared
// memory next to the tile.
__device__ __forceinline__ float tab_g(const float* t, int i) { return t[((i >> 2) << 3) + (i & 3)]; }
__device__ __forceinline__ float tab_inv(const float* t, int i) { return t[((i >> 2) << 3) + 4 + (i & 3)]; }
__device__ __forceinline__ float4 tab_g4(const float* t, int q) { return *reinterpret_cast<const float4*>(t + (q << 3)); }
__device__ __forceinline__ float4 tab_inv4(const float* t, int q)
{
    return *reinterpret_cast<const float4*>(t + (q << 3) + 4);
}

// One chunk of the forward / backward pass (positions 4q..4q+3): all four,
// or those with place u in [lo, hi] at the ends of the line.
__device__ __forceinline__ float fwd1(float g, float iv, float d, float& v)
{
    d = fmaf(g, d, v * iv);
    v = d;
    return d;
}
__device__ __forceinline__ float bwd1(float g, float x, float& v)
{
    x = fmaf(g, x, v);
    v = x;
    return x;
}
__device__ __forceinline__ float fwd4(float4& v, float4 g, float4 iv, float d)
{
    d = fwd1(g.x, iv.x, d, v.x);
    d = fwd1(g.y, iv.y, d, v.y);
    d = fwd1(g.z, iv.z, d, v.z);
    return fwd1(g.w, iv.w, d, v.w);
}
__device__ __forceinline__ float bwd4(float4& v, float4 g, float x)
{
    x = bwd1(g.w, x, v.w);
    x = bwd1(g.z, x, v.z);
    x = bwd1(g.y, x, v.y);
    return bwd1(g.x, x, v.x);
}
__device__ __forceinline__ float fwd4p(float4& v, float4 g, float4 iv, float d, int lo, int hi)
{
    if (lo <= 0 && 0 <= hi) d = fwd1(g.x, iv.x, d, v.x);
    if (lo <= 1 && 1 <= hi) d = fwd1(g.y, iv.y, d, v.y);
    if (lo <= 2 && 2 <= hi) d = fwd1(g.z, iv.z, d, v.z);
    if (lo <= 3 && 3 <= hi) d = fwd1(g.w, iv.w, d, v.w);
    return d;
}
__device__ __forceinline__ float bwd4p(float4& v, float4 g, float x, int lo, int hi)
{
    if (lo <= 3 && 3 <= hi) x = bwd1(g.w, x, v.w);
    if (lo <= 2 && 2 <= hi) x = bwd1(g.z, x, v.z);
    if (lo <= 1 && 1 <= hi) x = bwd1(g.y, x, v.y);
    if (lo <= 0 && 0 <= hi) x = bwd1(g.x, x, v.x);
    return x;
}

// Both passes of one line over positions 1..n-2 (n >= 3), chunk by chunk:
// ld(q) returns chunk q (positions 4q..4q+3) from shared memory and st(q, v)
// writes it back.  The two end chunks are peeled off, so the main loops run
// over whole chunks with no per-position tests; each loop keeps the next
// chunk and its coefficients loaded while the current chunk's dependent
// FFMAs run.  Only chunks up to the one holding position n - 2 are touched;
// places past the line's end in that chunk are written back unchanged.
template <class LD, class ST>
__device__ __forceinline__ void thomas_line(const float* t, int n, LD ld, ST st)
{
    const int ql = (n - 2) >> 2;      // chunk of position n - 2
    const int hl = n - 2 - 4 * ql;    // its place in that chunk
    // forward: chunk 0 (from position 1), whole chunks 1..ql-1, chunk ql
    float d = 0.f;
    {
        float4 v0 = ld(0);
        if (ql == 0) {
            d = fwd4p(v0, tab_g4(t, 0), tab_inv4(t, 0), d, 1, hl);
            st(0, v0);
        } else {
            float4 a = ld(1), ga = tab_g4(t, 1), ia = tab_inv4(t, 1);
            d = fwd4p(v0, tab_g4(t, 0), tab_inv4(t, 0), d, 1, 3);
            st(0, v0);
            int q = 1;   // a holds chunk q
            for (; q + 1 < ql; q += 2) {
                float4 b = ld(q + 1), gb = tab_g4(t, q + 1), ib = tab_inv4(t, q + 1);
                d = fwd4(a, ga, ia, d);
                st(q, a);
                a = ld(q + 2);
                ga = tab_g4(t, q + 2);
                ia = tab_inv4(t, q + 2);
                d = fwd4(b, gb, ib, d);
                st(q + 1, b);
            }
            if (q < ql) {   // q == ql - 1: one whole chunk, then chunk ql
                float4 b = ld(ql), gb = tab_g4(t, ql), ib = tab_inv4(t, ql);
                d = fwd4(a, ga, ia, d);
                st(q, a);
                d = fwd4p(b, gb, ib, d, 0, hl);
                st(ql, b);
            } else {        // a holds chunk ql
                d = fwd4p(a, ga, ia, d, 0, hl);
                st(ql, a);
            }
        }
    }
    // backward: chunk ql, whole chunks ql-1..1, chunk 0 (down to position 1)
    float x = 0.f;
    if (ql == 0) {
        float4 w = ld(0);
        x = bwd4p(w, tab_g4(t, 0), x, 1, hl);
        st(0, w);
        return;
    }
    float4 a = ld(ql), ga = tab_g4(t, ql);
    int q = ql;
    {
        float4 b = ld(q - 1), gb = tab_g4(t, q - 1);
        x = bwd4p(a, ga, x, 0, hl);
        st(q, a);
        a = b;
        ga = gb;
        --q;
    }
    for (; q - 1 >= 1; q -= 2) {   // a holds whole chunk q
        float4 b = ld(q - 1), gb = tab_g4(t, q - 1);
        x = bwd4(a, ga, x);
        st(q, a);
        a = ld(q - 2);
        ga = tab_g4(t, q - 2);
        x = bwd4(b, gb, x);
        st(q - 1, b);
    }
    if (q >= 1) {   // q == 1
        float4 b = ld(0), gb = tab_g4(t, 0);
        x = bwd4(a, ga, x);
        st(1, a);
        x = bwd4p(b, gb, x, 1, 3);
        st(0, b);
    } else {        // a holds chunk 0
        x = bwd4p(a, ga, x, 1, 3);
        st(0, a);
    }
}

// x tile through the row tensor map: lane t solves line t stored at
// st + t * P, P = row_smem_pitch(n).  All lanes sit at the same position, so
// the coefficients are one broadcast load, and each lane moves 4 values with
// one 16-byte shared access; P / 4 is odd, so the 8 lanes of each quarter
// warp hit 8 different 16-byte bank groups (no conflicts).
__device__ __forceinline__ void row_line(float* row, const LineRule& r, const float* t)
{
    const int n = static_cast<int>(r.n);
    if (n >= 3) {
        row[1] += r.fold;
        if (n > 3) row[n - 2] += r.fold;
        thomas_line(
            t, n, [row](int q) { return *reinterpret_cast<const float4*>(row + 4 * q); },
            [row](int q, float4 v) { *reinterpret_cast<float4*>(row + 4 * q) = v; });
    }
    if (r.dir) {
        row[0] = r.T;
        row[n - 1] = r.T;
    }
}

__device__ __forceinline__ void solve_rows_vec(float* st, const LineRule& r, const float* t, int lane,
                                               int count)
{
    if (lane >= count) return;
    row_line(st + lane * static_cast<int>(row_smem_pitch(r.n)), r, t);
}

// y/z tile: lane = column, rows at st + j * 32 (32 lanes, 32 banks).
__device__ __forceinline__ void solve_cols(float* st, const SweepTile& tile, const LineRule& r,
                                           const float* t, int lane, bool apply_faces)
{
    if (lane_col(tile, lane) >= tile.count || lane_slab(tile, lane) >= tile.nslab) return;
    const int n = static_cast<int>(r.n);
    float* c = st + lane;
    if (apply_faces && (tile.face & TILE_FACE) && on_face(tile, lane)) {
        for (int j = 0; j < n; ++j) c[j * 32] = r.T;   // applyDirichletBC fused: the line lies on a face
        return;
    }
    if (n >= 3) {
        c[32] += r.fold;
        if (n > 3) c[(n - 2) * 32] += r.fold;
        thomas_line(
            t, n,
            [c](int q) {
                return make_float4(c[(4 * q) * 32], c[(4 * q + 1) * 32], c[(4 * q + 2) * 32], c[(4 * q + 3) * 32]);
            },
            [c](int q, float4 v) {
                c[(4 * q) * 32] = v.x;
                c[(4 * q + 1) * 32] = v.y;
                c[(4 * q + 2) * 32] = v.z;
                c[(4 * q + 3) * 32] = v.w;
            });
    }
    if (r.dir) {
        c[0] = r.T;
        c[(n - 1) * 32] = r.T;
    }
}

// x tile moved as one 1-D bulk copy (lines longer than a tensor box): lane t
// solves line t stored at st + t * px.  Lane t reaches interior position i
// at step i + t, so at every step the 32 lanes touch 32 different banks
// (px is a multiple of 4, so px - 1 is odd).
__device__ __forceinline__ void skew_step_fwd(float* p, const float* t, int i, float& d)
{
    d = fmaf(tab_g(t, i + 1), d, p[i] * tab_inv(t, i + 1));
    p[i] = d;
}
__device__ __forceinline__ void skew_step_bwd(float* p, const float* t, int i, float& x)
{
    x = fmaf(tab_g(t, i + 1), x, p[i]);
    p[i] = x;
}

__device__ __forceinline__ void solve_rows(float* st, const SweepTile& tile, const LineRule& r, const float* t,
                                           int lane)
{
    const int n = static_cast<int>(r.n);
    const int px = static_cast<int>(tile.rs);
    const bool act = lane < static_cast<int>(tile.count);
    float* row = st + lane * px;
    if (n >= 3) {
        const int m = n - 2;
        float* p = row + 1;   // interior position i + 1 at p[i]
        if (act) {
            p[0] += r.fold;
            if (m > 1) p[m - 1] += r.fold;
        }
        // steps [0, 31) and [max(m, 31), m + 31) are predicated, [31, m) is
        // taken by every lane
        const int c_begin = m > 31 ? m : 31;
        float d = 0.f;
        for (int k = 0; k < 31; ++k) {
            const int i = k - lane;
            if (i >= 0 && i < m) skew_step_fwd(p, t, i, d);
        }
#pragma unroll 4
        for (int k = 31; k < m; ++k) skew_step_fwd(p, t, k - lane, d);
        for (int k = c_begin; k < m + 31; ++k) {
            const int i = k - lane;
            if (i >= 0 && i < m) skew_step_fwd(p, t, i, d);
        }
        float x = 0.f;
        for (int k = 0; k < 31; ++k) {
            const int i = m - 1 - (k - lane);
            if (i >= 0 && i < m) skew_step_bwd(p, t, i, x);
        }
#pragma unroll 4
        for (int k = 31; k < m; ++k) skew_step_bwd(p, t, m - 1 - (k - lane), x);
        for (int k = c_begin; k < m + 31; ++k) {
            const int i = m - 1 - (k - lane);
            if (i >= 0 && i < m) skew_step_bwd(p, t, i, x);
        }
    }
    if (act && r.dir) {
        row[0] = r.T;
        row[n - 1] = r.T;
    }
}

// ------------------------------------------------------------------ pipelined kernel

// Shared memory: kBarBytes of mbarriers ([warp][stage]), then the stages
// ([warp][stage][stage_floats], 128-byte aligned).  Between them, one tile
// descriptor per stage ([warp][stage], 64 bytes): the descriptor of the tile
// a stage holds, stashed when its load is issued.  Both regions are sized
// for the launch shape and rounded to 128 bytes.
constexpr int kBarBytes = 512;    // at most 16 warps x 4 stages
__host__ __device__ constexpr int round128(int b) { return (b + 127) & ~127; }
__host__ __device__ constexpr int sweep_bar_bytes(int warps, int nstages) { return round128(warps * nstages * 8); }
__host__ __device__ constexpr int sweep_header_bytes(int warps, int nstages)
{
    return sweep_bar_bytes(warps, nstages) + round128(warps * nstages * 64);
}

template <bool kRows>
__global__ void __launch_bounds__(256, 1) k_sweep_tma(float* __restrict__ dens, const SweepTile* __restrict__ tiles,
                                                   uint32_t ntiles, const float* __restrict__ tab,
                                                   const void* __restrict__ tmaps, int stage_floats, int nstages,
                                                   int tab_area, int apply_faces,
                                                   const uint8_t* __restrict__ mask, unsigned* __restrict__ status)
{
    // stage: [tile data][tab_area floats of coefficient table]
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem) + warp * nstages;
    SweepTile* descs = reinterpret_cast<SweepTile*>(smem + sweep_bar_bytes(nwarps, nstages)) + warp * nstages;
    float* stages = reinterpret_cast<float*>(smem + sweep_header_bytes(nwarps, nstages)) +
                    static_cast<size_t>(warp) * nstages * stage_floats;
    if (lane == 0)
        for (int s = 0; s < nstages; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncwarp();

    const uint32_t gw = blockIdx.x * nwarps + warp, tw = gridDim.x * nwarps;
    const uint32_t ntw = gw < ntiles ? (ntiles - gw + tw - 1) / tw : 0u;
    const int ahead = nstages - 1;   // loads in flight while one stage is solved
    uint32_t issued = 0;
    bool ok = true;
    // 'nd' is the descriptor of the next tile to issue, loaded one tile
    // ahead so its latency hides behind the current solve
    SweepTile nd{};
    if (ntw) nd = tiles[gw];
    auto issue = [&]() {
        const int s = static_cast<int>(issued % nstages);
        float* st = stages + s * stage_floats;
        issue_tile_load<kRows>(nd, dens, tab, tmaps, st, st + stage_floats - tab_area, &bars[s], lane, status);
        if (lane == 0) descs[s] = nd;
        ++issued;
        if (issued < ntw) nd = tiles[gw + issued * tw];
    };
    while (issued < ntw && static_cast<int>(issued) < ahead) issue();
    for (uint32_t k = 0; k < ntw; ++k) {
        // refill: tile k + ahead goes to the stage of tile k - 1, whose store
        // (issued last) must have finished reading shared memory
        if (issued < ntw) {
            bulk_wait_read<0>();
            __syncwarp();
            issue();
        }
        const int s = static_cast<int>(k % nstages);
        if (!mbar_wait(&bars[s], (k / nstages) & 1u, status)) {
            ok = false;
            break;
        }
        __syncwarp();
        const SweepTile tile = descs[s];
        const LineRule r = rule_of(tile);
        float* st = stages + s * stage_floats;
        const float* t = st + stage_floats - tab_area;
        if (tile_on(r, mask)) {
            if (kRows) {
                if (tile.face & TILE_TENSOR) solve_rows_vec(st, r, t, lane, static_cast<int>(tile.count));
                else solve_rows(st, tile, r, t, lane);
            } else {
                solve_cols(st, tile, r, t, lane, apply_faces != 0);
            }
        }
        fence_async_smem();
        __syncwarp();
        issue_tile_store<kRows>(tile, dens, tmaps, st, lane);
    }
    if (!ok) {
        // let every load this warp issued land before the CTA exits (bounded)
        for (uint32_t k = 0; k < issued; ++k) {
            const int s = static_cast<int>(k % nstages);
            if (!mbar_wait(&bars[s], (k / nstages) & 1u, status)) break;
        }
    }
    bulk_wait_all();
}

// ------------------------------------------------------- fused x + y sweeps of a plane

// Column line of a plane in shared memory (rows P floats apart): the steps
// of solve_cols with row stride P.  'face': the line lies on an x face of a
// 2-D block whose last sweep this is, so applyDirichletBC sets it to T.
__device__ __forceinline__ void plane_col(float* c, int P, const LineRule& r, const float* t, bool face)
{
    const int n = static_cast<int>(r.n);
    if (face) {
        for (int j = 0; j < n; ++j) c[j * P] = r.T;
        return;
    }
    if (n >= 3) {
        c[P] += r.fold;
        if (n > 3) c[(n - 2) * P] += r.fold;
        auto ld = [c, P](int q) {
            return make_float4(c[(4 * q) * P], c[(4 * q + 1) * P], c[(4 * q + 2) * P], c[(4 * q + 3) * P]);
        };
        auto st4 = [c, P](int q, float4 v) {
            c[(4 * q) * P] = v.x;
            c[(4 * q + 1) * P] = v.y;
            c[(4 * q + 2) * P] = v.z;
            c[(4 * q + 3) * P] = v.w;
        };
        thomas_line(t, n, ld, st4);
    }
    if (r.dir) {
        c[0] = r.T;
        c[(n - 1) * P] = r.T;
    }
}

// One CTA per x-y plane (one z slab of one instance-substrate): the plane
// (rows of pitch P = row_smem_pitch(nx), zero-filled past nx) and both
// rules' tables come in with one tensor box and two bulk copies; every row
// is solved (x sweep), then every column (y sweep), and the plane goes back
// with one tensor store.  The steps on each line are those of the x and y
// tile kernels, so the result is the same bits, but the plane crosses HBM
// once for both sweeps.  Several CTAs per SM overlap one plane's copies
// with another's solves, and each CTA prefetches into L2 (a tensor-box
// prefetch, no shared memory) the plane of the CTA 'ahead' jobs later, so
// that CTA's load is served from L2.
__global__ void __launch_bounds__(kPlaneThreads) k_sweep_planes(const PlaneJob* __restrict__ jobs,
                                                                const float* __restrict__ tab,
                                                                const void* __restrict__ tmaps, int apply_faces,
                                                                const uint8_t* __restrict__ mask,
                                                                unsigned* __restrict__ status, uint32_t ahead)
{
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    float* pl = reinterpret_cast<float*>(smem + 128);
    const PlaneJob jb = jobs[blockIdx.x];
    const uint32_t ii = jb.inst & kPlaneInstMask;
    if (mask && !(mask[ii] & STEP_DIFFUSE)) return;   // the whole CTA leaves together
    const bool zk = (jb.inst & kPlaneZ) != 0;
    const uint32_t nx = jb.nx, ny = jb.ny, P = plane_pitch(nx, zk);
    float* tx = pl + plane_data_floats(nx, ny, zk);
    float* ty = zk ? tx : tx + tab_floats(nx);
    const void* map = static_cast<const unsigned char*>(tmaps) + static_cast<size_t>(jb.map) * 128;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t tbx = zk ? 0u : tab_floats(nx) * 4u, tby = tab_floats(ny) * 4u;
        mbar_arrive_expect_tx(bar, P * ny * 4u + tbx + tby);   // the whole box, fill included
        if (zk) {
            tensor_load3(pl, map, 0, static_cast<int>(jb.row0), 0, bar);
        } else {
            tensor_load2(pl, map, 0, static_cast<int>(jb.row0), bar);
            bulk_load(tx, tab + jb.tab_x, tbx, bar);
        }
        bulk_load(ty, tab + jb.tab_y, tby, bar);
        // the plane of a CTA that starts a little later ('ahead' jobs on,
        // about a quarter of a residency): into L2 now, so its load is an
        // L2 hit rather than a wait on HBM
        if (ahead != 0 && blockIdx.x + ahead < gridDim.x) {
            const PlaneJob nj = jobs[blockIdx.x + ahead];
            if (!mask || (mask[nj.inst & kPlaneInstMask] & STEP_DIFFUSE)) {
                const void* nmap = static_cast<const unsigned char*>(tmaps) + static_cast<size_t>(nj.map) * 128;
                if (nj.inst & kPlaneZ) tensor_prefetch3(nmap, 0, static_cast<int>(nj.row0), 0);
                else tensor_prefetch2(nmap, 0, static_cast<int>(nj.row0));
            }
        }
    }
    bool got;
    if (status[1] & PCG_DEV_TEST_GIVE_UP) {   // test switch: this wait's bound ran out
        if (threadIdx.x == 0) atomicOr(status, PCG_DEV_TIMEOUT);
        got = false;
    } else {
        got = mbar_wait(bar, 0, status);
    }
    if (!__syncthreads_and(got)) {
        // a wait ran out: one more bounded wait for the copies before the
        // CTA releases its shared memory
        if (threadIdx.x == 0 && !got) mbar_wait(bar, 0, status);
        return;
    }
    LineRule rx{}, ry{};
    rx.n = nx;
    rx.fold = jb.fold_x;
    rx.T = jb.T_x;
    rx.dir = (jb.inst & kPlaneDirX) ? 1u : 0u;
    ry.n = ny;
    ry.fold = jb.fold_y;
    ry.T = jb.T_y;
    ry.dir = (jb.inst & kPlaneDirY) ? 1u : 0u;
    if (!zk) {
        for (uint32_t r = threadIdx.x; r < ny; r += blockDim.x) row_line(pl + r * P, rx, tx);
        __syncthreads();
    }
    // faces of the block's last sweep (2-D: y, 3-D: z): x faces, and a whole
    // z plane on a y face
    const bool faces = apply_faces && (jb.inst & kPlaneFaces) != 0;
    const bool slab_face = (jb.inst & kPlaneSlabFace) != 0;
    for (uint32_t c = threadIdx.x; c < nx; c += blockDim.x)
        plane_col(pl + c, static_cast<int>(P), ry, ty, faces && (slab_face || c == 0u || c + 1u == nx));
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
        if (zk) tensor_store3(map, 0, static_cast<int>(jb.row0), 0, pl);
        else tensor_store2(map, 0, static_cast<int>(jb.row0), pl);
        bulk_commit();
        bulk_wait_read<0>();   // shared memory may be released once the store has read it
    }
}

// ------------------------------------------------------- any line length

// Reference rule for a whole line held at s[m * st], sequentially (lines
// longer than the shared-memory tiles).
__device__ __forceinline__ void solve_line(float* s, size_t st, const LineRule& r, const float* __restrict__ t)
{
    const int n = static_cast<int>(r.n);
    if (n >= 3) {
        float d = 0.f;
        for (int i = 1; i <= n - 2; ++i) {
            const float f = (i == 1 || i == n - 2) ? r.fold : 0.f;
            d = fmaf(__ldg(t + ((i >> 2) << 3) + (i & 3)), d, (s[i * st] + f) * __ldg(t + ((i >> 2) << 3) + 4 + (i & 3)));
            s[i * st] = d;
        }
        float x = 0.f;
        for (int i = n - 2; i >= 1; --i) {
            x = fmaf(__ldg(t + ((i >> 2) << 3) + (i & 3)), x, s[i * st]);
            s[i * st] = x;
        }
    }
    if (r.dir) {
        s[0] = r.T;
        s[(n - 1) * st] = r.T;
    }
}

__global__ void __launch_bounds__(128) k_sweep_global(float* __restrict__ dens, const SweepTile* __restrict__ tiles,
                                                      uint32_t ntiles,
                                                      const float* __restrict__ tab, int apply_faces,
                                                      const uint8_t* __restrict__ mask)
{
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = gw; t < ntiles; t += nw) {
        const SweepTile tile = tiles[t];
        if (static_cast<uint32_t>(lane) >= tile.count) continue;
        const LineRule r = rule_of(tile);
        if (!tile_on(r, mask)) continue;
        const bool rows = (tile.face & TILE_ROWS) != 0;
        // row tiles: lines tile.rs apart, unit stride; column tiles: adjacent lines, stride tile.rs
        float* g = dens + tile.base + (rows ? static_cast<size_t>(lane) * tile.rs : static_cast<size_t>(lane));
        const size_t st = rows ? 1 : tile.rs;
        if (!rows && apply_faces && (tile.face & TILE_FACE) && on_face(tile, lane)) {
            for (uint32_t j = 0; j < r.n; ++j) g[j * st] = r.T;
        } else {
            solve_line(g, st, r, tab + r.tab);
        }
    }
}

// ------------------------------------------------------------- Dirichlet

__global__ void k_dirichlet(float* __restrict__ dens, const FaceJob* __restrict__ jobs)
{
    const FaceJob jb = jobs[blockIdx.x];
    float* base = dens + jb.base;
    const uint32_t nx = jb.nx, ny = jb.ny, nz = jb.nz;
    const size_t px = jb.px, slab = px * ny;
    // edges of every slab (microenvironment.mm:140-150)
    const uint32_t per = 2u * nx + 2u * ny;
    const size_t total = static_cast<size_t>(nz) * per;
    for (size_t e = threadIdx.x; e < total; e += blockDim.x) {
        const uint32_t k = static_cast<uint32_t>(e / per), q = static_cast<uint32_t>(e % per);
        uint32_t i, j;
        if (q < nx) { i = q; j = 0; }
        else if (q < 2u * nx) { i = q - nx; j = ny - 1; }
        else if (q < 2u * nx + ny) { i = 0; j = q - 2u * nx; }
        else { i = nx - 1; j = q - 2u * nx - ny; }
        base[k * slab + j * px + i] = jb.T;
    }
    if (nz > 1) {   // z faces (3-D rule)
        const size_t plane = static_cast<size_t>(nx) * ny;
        for (size_t e = threadIdx.x; e < 2 * plane; e += blockDim.x) {
            const size_t k = (e < plane) ? 0 : (nz - 1);
            const size_t v = e % plane;
            base[k * slab + (v / nx) * px + (v % nx)] = jb.T;
        }
    }
}

// ------------------------------------------------------------- gradients

__global__ void k_gradients(const float* __restrict__ dens, float* __restrict__ gx, float* __restrict__ gy,
                            float* __restrict__ gz, const GradJob* __restrict__ jobs)
{
    const GradJob jb = jobs[blockIdx.y];
    const size_t nx = jb.nx, ny = jb.ny, nz = jb.nz, nv = nx * ny * nz, px = jb.px;
    const float* D = dens + jb.base;
    for (size_t n = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; n < nv;
         n += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t i = n % nx, j = (n / nx) % ny, k = n / (nx * ny);
        const size_t a = (k * ny + j) * px + i;       // device offset of voxel n
        const size_t o = jb.out_base + n;             // dense output
        const size_t sy = px, sz = px * ny;
        double v;
        if (nx == 1) v = 0.0;
        else if (i == 0) v = (static_cast<double>(D[a + 1]) - D[a]) * jb.inv_dx;
        else if (i == nx - 1) v = (static_cast<double>(D[a]) - D[a - 1]) * jb.inv_dx;
        else v = (static_cast<double>(D[a + 1]) - D[a - 1]) * 0.5 * jb.inv_dx;
        if (gx) gx[o] = static_cast<float>(v);
        if (ny == 1) v = 0.0;
        else if (j == 0) v = (static_cast<double>(D[a + sy]) - D[a]) * jb.inv_dy;
        else if (j == ny - 1) v = (static_cast<double>(D[a]) - D[a - sy]) * jb.inv_dy;
        else v = (static_cast<double>(D[a + sy]) - D[a - sy]) * 0.5 * jb.inv_dy;
        if (gy) gy[o] = static_cast<float>(v);
        if (nz > 1) {
            if (k == 0) v = (static_cast<double>(D[a + sz]) - D[a]) * jb.inv_dz;
            else if (k == nz - 1) v = (static_cast<double>(D[a]) - D[a - sz]) * jb.inv_dz;
            else v = (static_cast<double>(D[a + sz]) - D[a - sz]) * 0.5 * jb.inv_dz;
        } else {
            v = 0.0;
        }
        if (gz) gz[o] = static_cast<float>(v);
    }
}

// ------------------------------------------------------------- launchers

size_t sweep_tma_smem(int warps, int nstages, int stage_floats)
{
    return static_cast<size_t>(sweep_header_bytes(warps, nstages)) +
           static_cast<size_t>(warps) * nstages * stage_floats * sizeof(float);
}

static cudaError_t allow_max_smem(const void* fn)
{
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    return e;
}

int sweep_tma_occupancy(bool rows, int warps, int nstages, int stage_floats)
{
    const void* fn = rows ? reinterpret_cast<const void*>(k_sweep_tma<true>)
                          : reinterpret_cast<const void*>(k_sweep_tma<false>);
    if (warps < 1 || warps * nstages * 8 > kBarBytes || nstages < 2) return 0;
    if (allow_max_smem(fn) != cudaSuccess) return 0;
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, warps * 32, sweep_tma_smem(warps, nstages, stage_floats)) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return b;
}

cudaError_t launch_sweep_tma(cudaStream_t st, bool rows, float* dens, const SweepTile* tiles, uint32_t ntiles,
                             const float* tab, const void* tmaps, int apply_faces,
                             const uint8_t* mask, unsigned* status, TmaCfg cfg)
{
    if (ntiles == 0) return cudaSuccess;
    // stages start 128-byte aligned (tensor copies), the table area on 32 bytes
    if (cfg.stage_floats % 32 != 0 || cfg.tab_floats % 8 != 0 || cfg.tab_floats >= cfg.stage_floats)
        return cudaErrorInvalidValue;
    const size_t smem = sweep_tma_smem(cfg.warps, cfg.stages, cfg.stage_floats);
    if (rows)
        k_sweep_tma<true><<<cfg.grid, cfg.warps * 32, smem, st>>>(dens, tiles, ntiles, tab, tmaps,
                                                                   cfg.stage_floats, cfg.stages, cfg.tab_floats,
                                                                   apply_faces, mask, status);
    else
        k_sweep_tma<false><<<cfg.grid, cfg.warps * 32, smem, st>>>(dens, tiles, ntiles, tab, tmaps,
                                                                    cfg.stage_floats, cfg.stages, cfg.tab_floats,
                                                                    apply_faces, mask, status);
    return cudaGetLastError();
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependency on libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        cudaGetLastError();
    }
    return fn;
}

bool encode_column_map(void* map128, float* block, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t px, int axis,
                       uint32_t n, uint32_t width)
{
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || n == 0 || n > kTensorMaxN || (px & 3u) || (reinterpret_cast<uintptr_t>(block) & 15u)) return false;
    if (width != 32u && width != 16u && width != 8u) return false;
    const cuuint64_t row = static_cast<cuuint64_t>(px) * 4u, slab = row * ny;
    // y lines: (x, z, y); z lines: (x, y, z) -- the line runs along the last dimension
    const cuuint64_t dims[3] = {nx, axis == 1 ? nz : ny, axis == 1 ? ny : nz};
    const cuuint64_t strides[2] = {axis == 1 ? slab : row, axis == 1 ? row : slab};
    const cuuint32_t box[3] = {width, 32u / width, n};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    const CUresult r = fn(static_cast<CUtensorMap*>(map128), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, block, dims, strides,
                          box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool encode_row_map(void* map128, float* block, uint32_t nx, uint64_t rows, uint32_t px)
{
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    const uint32_t P = row_smem_pitch(nx);
    if (!fn || nx == 0 || nx > kRowTensorMaxN || rows == 0 || (px & 3u) || px < nx ||
        (reinterpret_cast<uintptr_t>(block) & 15u))
        return false;
    const cuuint64_t dims[2] = {nx, rows};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(px) * 4u};
    const cuuint32_t box[2] = {P, 32u};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = fn(static_cast<CUtensorMap*>(map128), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, block, dims, strides,
                          box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool encode_plane_map(void* map128, float* block, uint32_t nx, uint32_t ny, uint64_t rows, uint32_t px)
{
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    const uint32_t P = row_smem_pitch(nx);
    if (!fn || nx == 0 || nx > kRowTensorMaxN || ny == 0 || ny > 256 || rows == 0 || (px & 3u) || px < nx ||
        (reinterpret_cast<uintptr_t>(block) & 15u))
        return false;
    const cuuint64_t dims[2] = {nx, rows};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(px) * 4u};
    const cuuint32_t box[2] = {P, ny};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = fn(static_cast<CUtensorMap*>(map128), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, block, dims, strides,
                          box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// x-z planes of one instance-substrate for the z lines: dims (x, y, z), box
// round4(nx) x 1 x nz (the full x extent, one y, every z).
bool encode_xz_plane_map(void* map128, float* block, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t px)
{
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    const uint32_t bx = (nx + 3u) & ~3u;
    if (!fn || nx == 0 || bx > 256 || nz == 0 || nz > 256 || ny == 0 || (px & 3u) || px < nx ||
        (reinterpret_cast<uintptr_t>(block) & 15u))
        return false;
    const cuuint64_t row = static_cast<cuuint64_t>(px) * 4u;
    const cuuint64_t dims[3] = {nx, ny, nz};
    const cuuint64_t strides[2] = {row, row * ny};
    const cuuint32_t box[3] = {bx, 1u, nz};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    const CUresult r = fn(static_cast<CUtensorMap*>(map128), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, block, dims, strides,
                          box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

size_t sweep_planes_smem(uint32_t floats) { return 128 + static_cast<size_t>(floats) * sizeof(float); }

cudaError_t sweep_planes_prepare()
{
    const void* fn = reinterpret_cast<const void*>(k_sweep_planes);
    cudaError_t e = allow_max_smem(fn);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    return e;
}

int sweep_planes_ctas(uint32_t floats)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sweep_planes, kPlaneThreads, sweep_planes_smem(floats)) !=
        cudaSuccess)
        return 0;
    return n;
}

cudaError_t launch_sweep_planes(cudaStream_t st, const PlaneJob* jobs, uint32_t njobs, const float* tab,
                                const void* tmaps, uint32_t floats, int apply_faces, const uint8_t* mask,
                                unsigned* status)
{
    if (njobs == 0) return cudaSuccess;
    // prefetch distance: a quarter of the CTAs of this launch resident at
    // once (measured: a half, one or two residencies ahead gain less or lose).
    // The SM count is read once, on the first device used; it only sets this
    // distance, never which data is read.
    static const int sms = [] {
        int dev = 0, n = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            n = 1;
        return n;
    }();
    const uint32_t ahead = static_cast<uint32_t>(sweep_planes_ctas(floats) * sms / 4);
    k_sweep_planes<<<njobs, kPlaneThreads, sweep_planes_smem(floats), st>>>(jobs, tab, tmaps, apply_faces, mask,
                                                                            status, ahead);
    return cudaGetLastError();
}

cudaError_t launch_sweep_global(cudaStream_t st, float* dens, const SweepTile* tiles, uint32_t ntiles,
                                const float* tab, int apply_faces, const uint8_t* mask,
                                int grid)
{
    if (ntiles == 0) return cudaSuccess;
    k_sweep_global<<<grid, 128, 0, st>>>(dens, tiles, ntiles, tab, apply_faces, mask);
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
