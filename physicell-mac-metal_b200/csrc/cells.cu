// cells.cu — per-cell kernels (sm_100a): secretion/uptake, spatial binning,
// sorted SoA, neighbour forces and the Adams-Bashforth update.
//
// Reference semantics:
//   secretion  src/cell_phenotype.cpp:526-564 (processSecretion), FP64 per
//              cell, FP32 density store after every cell;
//   binning    shaders/mechanics.metal:54-76 (FP32 divide + truncation);
//   forces     shaders/mechanics.metal:91-216;
//   integrate  shaders/integrate.metal:31-80, clamp box = mechanics grid
//              (src/cell_mechanics.mm:57-70);
//   voxel refresh  Microenvironment::voxelIndex (microenvironment.mm:176-184).
// The reference's GPU hash and CPU secretion loop are racy; here every
// result is deterministic: for secretion, cells are sorted by (diffusion
// voxel, cell index) (secorder.cu) and each voxel's cells are applied in
// that order; the mechanics binning is a counting sort whose
// order within a voxel is fixed by ranks (index, and x for the force
// pass), so every cell's neighbour walk and sum have a fixed order.
#include "pcg_kernels.cuh"

namespace pcg {

__device__ __forceinline__ uint32_t fbits(float f) { return __float_as_uint(f); }

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// (int)((p - lo) / h) with IEEE FP32 subtract and divide; cvt.rzi saturates
// out-of-range values and maps NaN to 0.
__device__ __forceinline__ int bin_of(float p, float lo, float h)
{
    return __float2int_rz(__fdiv_rn(__fsub_rn(p, lo), h));
}

// ------------------------------------------------------------------ secretion

// Secretion constants of every cell, in cell order: for rate slot
// o = in.rate_off + (g - in.cell_off) * S + s, three arrays of n_rate,
// cc[{0,1,2} * n_rate + o] = {dt*ne/V_vox, ic*sec*sat, 1 + ic*(sec+upt)} with
// ic = dt*V_cell/V_vox, exactly as processSecretion forms them
// (cell_phenotype.cpp:526-564).  They change only with the rates, volumes,
// voxel size or dt; a new order only permutes them (k_sec_permute).
__global__ void k_sec_cell_consts(const float* __restrict__ soa, uint32_t stride, uint32_t n,
                                  const uint32_t* __restrict__ cell_inst, const CellInst* __restrict__ insts,
                                  const double* __restrict__ rates4, uint32_t n_rate, double dt,
                                  double* __restrict__ cc, uint32_t* __restrict__ flags)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = g < n;
    const unsigned live_lanes = __ballot_sync(0xFFFFFFFFu, live);   // blocks are whole warps
    if (!live) return;
    const uint32_t ii = cell_inst[g];
    const CellInst& in = insts[ii];
    const double V_vox = __dmul_rn(__dmul_rn(static_cast<double>(in.dx), static_cast<double>(in.dy)),
                                   static_cast<double>(in.dz));
    const double V_cell = static_cast<double>(soa[static_cast<size_t>(F_TOTAL_VOL) * stride + g]);
    const double ic = __ddiv_rn(__dmul_rn(dt, V_cell), V_vox);
    const uint32_t src = in.rate_off + (g - in.cell_off) * in.S;
    uint32_t f = 0;
    for (uint32_t s = 0; s < in.S; ++s) {
        const uint32_t o = src + s;
        const double sec = rates4[o], upt = rates4[n_rate + o], sat = rates4[2ull * n_rate + o],
                     ne = rates4[3ull * n_rate + o];
        const double c0 = __ddiv_rn(__dmul_rn(dt, ne), V_vox);
        const double c1 = __dmul_rn(__dmul_rn(ic, sec), sat);
        cc[o] = c0;
        cc[static_cast<uint64_t>(n_rate) + o] = c1;
        cc[2ull * n_rate + o] = __dadd_rn(1.0, __dmul_rn(ic, __dadd_rn(sec, upt)));
        f |= (__double_as_longlong(c0) != 0 ? 1u : 0u) | (__double_as_longlong(c1) != 0 ? 2u : 0u);
    }
    // per instance: does any cell have an export (bit 0) or a secretion
    // (bit 1) term other than +0?  Cells of a warp mostly share the instance.
    // (A cell outside the sorted order may set a bit: the secretion pass
    // then reads that instance's stored terms, which give the same bits.)
    const unsigned grp = __match_any_sync(live_lanes, ii);
    f = __reduce_or_sync(grp, f);
    if (f && (threadIdx.x & 31) == static_cast<unsigned>(__ffs(grp) - 1)) atomicOr(&flags[ii], f);
}

// The constants in sorted order: the cell sorder[q] of instance i goes to
// rate slot in.rate_off + (q - in.cell_off) * S (+ s) of the three arrays
// cs[{0,1,2} * n_rate + slot] (an instance's secreting cells fill the start
// of its range).  c0 and c1 are moved only for instances that have a term
// other than +0 (flags), the only ones the secretion pass reads them for.
__global__ void k_sec_permute(const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ sorder, uint32_t n,
                              const uint32_t* __restrict__ cell_inst, const CellInst* __restrict__ insts,
                              uint32_t invalid_key, const uint32_t* __restrict__ flags,
                              const double* __restrict__ cc, uint32_t n_rate, double* __restrict__ cs)
{
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    if (skeys[q] >= invalid_key) return;
    const uint32_t g = sorder[q];
    const uint32_t ii = cell_inst[g];
    const CellInst& in = insts[ii];
    const uint32_t f = flags[ii];
    const uint64_t src = in.rate_off + (g - in.cell_off) * in.S;
    const uint64_t dst = in.rate_off + (q - in.cell_off) * in.S;
    for (uint32_t s = 0; s < in.S; ++s) {
        if (f & 1u) cs[dst + s] = cc[src + s];
        if (f & 2u) cs[n_rate + dst + s] = cc[n_rate + src + s];
        cs[2ull * n_rate + dst + s] = cc[2ull * n_rate + src + s];
    }
}

// One cell's processSecretion on one substrate (cell_phenotype.cpp:526-564):
// rho += c0; rho = (rho + c1) / c2; clamp at 0; FP32 store.  A term the
// instance never has (flags) is exactly +0 and is added as the constant.
__device__ __forceinline__ float secrete_terms(float rho32, double c0, double c1, double c2)
{
    double rho = static_cast<double>(rho32);
    rho = __dadd_rn(rho, c0);
    rho = __dadd_rn(rho, c1);
    rho = __ddiv_rn(rho, c2);
    if (rho < 0.0) rho = 0.0;
    return __double2float_rn(rho);
}

__device__ __forceinline__ float secrete_cell(float rho32, const double* __restrict__ cs, uint64_t o, uint64_t cap,
                                              uint32_t f)
{
    return secrete_terms(rho32, (f & 1u) ? cs[o] : 0.0, (f & 2u) ? cs[cap + o] : 0.0, cs[2 * cap + o]);
}

// One thread per run: applies the run's cells to its voxel in ascending
// cell index (the stable order), FP64 per cell with the FP32 store after
// each cell.  The run's metadata is read once; with one or two substrates
// both are held in registers and advanced together.  Constants: three
// arrays of cap (c0, c1, c2), entry (cell in sorted order, substrate).
__global__ void __launch_bounds__(256, 6) k_secrete(float* __restrict__ dens, const uint32_t* __restrict__ run_start,
                          const uint64_t* __restrict__ run_word, const uint32_t* __restrict__ n_runs,
                          const CellInst* __restrict__ insts, const double* __restrict__ cs, uint64_t cap,
                          const uint32_t* __restrict__ flags, const uint8_t* __restrict__ mask)
{
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= *n_runs) return;
    // a run's start and word (instance, the voxel's density element) were
    // placed when the order was built, so the density is one load away and
    // the first cell's rate slot one (cached) instance record away
    const uint64_t w = run_word[r];
    const uint32_t ii = static_cast<uint32_t>(w >> kRunDensBits);
    if (ii == kRunNone) return;   // the instance's non-secreting cells
    const uint32_t p0 = run_start[r], p1 = run_start[r + 1];
    float* d = dens + (w & kRunDensMask);
    if (mask && !(mask[ii] & STEP_DIFFUSE)) return;
    const CellInst& in = insts[ii];
    const uint64_t base = in.rate_off + (p0 - in.cell_off) * in.S;   // 32-bit slots, as the rates
    const uint32_t S = in.S;
    const uint32_t f = flags[ii];
    if (S <= 2) {
        // the first cell's terms and the voxel's densities in one batch of
        // independent loads (a loop would order the terms after the density)
        const bool two = S > 1;
        const double a0 = (f & 1u) ? cs[base] : 0.0, b0 = (f & 2u) ? cs[cap + base] : 0.0, c0 = cs[2 * cap + base];
        double a1 = 0.0, b1 = 0.0, c1 = 1.0;
        if (two) {
            a1 = (f & 1u) ? cs[base + 1] : 0.0;
            b1 = (f & 2u) ? cs[cap + base + 1] : 0.0;
            c1 = cs[2 * cap + base + 1];
        }
        float r0 = d[0], r1 = two ? d[in.sub_pitch] : 0.f;
        r0 = secrete_terms(r0, a0, b0, c0);
        if (two) r1 = secrete_terms(r1, a1, b1, c1);
        for (uint32_t q = p0 + 1; q < p1; ++q) {
            const uint64_t o = base + static_cast<uint64_t>(q - p0) * S;
            r0 = secrete_cell(r0, cs, o, cap, f);
            if (S > 1) r1 = secrete_cell(r1, cs, o + 1, cap, f);
        }
        d[0] = r0;
        if (S > 1) d[in.sub_pitch] = r1;
        return;
    }
    for (uint32_t s = 0; s < S; ++s, d += in.sub_pitch) {
        float rho32 = *d;
        for (uint32_t q = p0; q < p1; ++q)
            rho32 = secrete_cell(rho32, cs, base + static_cast<uint64_t>(q - p0) * S + s, cap, f);
        *d = rho32;
    }
}

// ------------------------------------------------------------------ removal

// The copies of a batch of CellData::removeCell calls (cell_data.cpp:408-
// 498): move m puts the cell at place src into place dst.  Every source lies
// at or past the new cell count and every destination before it, so no copy
// reads a place that another copy writes.  One thread per (move, item): the
// 28 SoA fields (copied as bits), the four per-substrate rate arrays, the
// active flag and the three FP64 master positions.
__global__ void k_cells_move(uint32_t* __restrict__ soa, uint32_t stride, const uint2* __restrict__ moves,
                             uint32_t n_moves, double* __restrict__ rates, uint64_t rate_cap, uint32_t S,
                             uint8_t* __restrict__ active, double* __restrict__ pos64)
{
    const uint32_t items = NUM_FIELDS + 4u * S + 1u + 3u;
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<uint64_t>(n_moves) * items) return;
    const uint32_t m = static_cast<uint32_t>(t / items), it = static_cast<uint32_t>(t % items);
    const uint32_t dst = moves[m].x, src = moves[m].y;
    if (it < static_cast<uint32_t>(NUM_FIELDS)) {
        soa[static_cast<size_t>(it) * stride + dst] = soa[static_cast<size_t>(it) * stride + src];
    } else if (it < NUM_FIELDS + 4u * S) {
        const uint32_t q = (it - NUM_FIELDS) / S, s = (it - NUM_FIELDS) % S;
        double* r = rates + q * rate_cap;
        r[static_cast<size_t>(dst) * S + s] = r[static_cast<size_t>(src) * S + s];
    } else if (it == NUM_FIELDS + 4u * S) {
        active[dst] = active[src];
    } else if (pos64) {
        const size_t a = it - (NUM_FIELDS + 4u * S + 1u);
        pos64[a * stride + dst] = pos64[a * stride + src];
    }
}

// ------------------------------------------------------------------ mechanics

// Binning is a counting sort over the mechanics voxels of the whole batch.
// k_mech_bin finds each cell's voxel (FP32 divide, truncation and clamp,
// as mechanics.metal:54-76) and counts it; the atomic's return value is the
// cell's arrival slot in its voxel.  The exclusive scan of the counts is the
// cell-start table.  k_mech_place drops each cell, with its x position, at
// start + slot, which groups the voxel's cells in arrival order, and
// k_mech_order ranks every cell in its voxel twice: by index (the stable
// order of the cell-start table, sorder: syncHashPointers' voxelCells) and
// by x position, index breaking ties (the force pass's order: the sorted
// positions and strengths, the cell's index riding in the strengths' third
// component, which the force terms never read).  Bins grow with x, so the
// cells of a run of voxels along x are in x order as a whole in the force
// order.  Every store is a scattered partial sector, and their rate bounds
// the kernel, so the stable order is only written where it is read
// (SORDER; a batch makes it on request, k_mech_stable_order) and the force
// order needs no index array of its own.
__global__ void k_mech_bin(float* __restrict__ soa, uint32_t stride, uint32_t n, const uint32_t* __restrict__ cell_inst,
                           const CellInst* __restrict__ insts, uint32_t* __restrict__ keys,
                           uint32_t* __restrict__ slots, uint32_t* __restrict__ counts,
                           const uint8_t* __restrict__ mask)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t ii = cell_inst[g];
    const CellInst& in = insts[ii];
    const float px = soa[static_cast<size_t>(F_POS_X) * stride + g];
    const float py = soa[static_cast<size_t>(F_POS_Y) * stride + g];
    const float pz = soa[static_cast<size_t>(F_POS_Z) * stride + g];
    const int vi = clampi(bin_of(px, in.mx_min, in.vs), 0, static_cast<int>(in.mnx) - 1);
    const int vj = clampi(bin_of(py, in.my_min, in.vs), 0, static_cast<int>(in.mny) - 1);
    const int vk = clampi(bin_of(pz, in.mz_min, in.vs), 0, static_cast<int>(in.mnz) - 1);
    const uint32_t local = static_cast<uint32_t>(vk) * in.mny * in.mnx + static_cast<uint32_t>(vj) * in.mnx +
                           static_cast<uint32_t>(vi);
    // every cell is binned (the sort covers the whole batch) but only the
    // instances taking this mechanics step store their bin
    if (mask == nullptr || (mask[ii] & STEP_MECH)) soa[static_cast<size_t>(F_MECH_VOXEL) * stride + g] = __uint_as_float(local);
    const uint32_t key = in.mvox_base + local;
    keys[g] = key;
    slots[g] = atomicAdd(&counts[key], 1u);
}

// Order-preserving map of FP32 bit patterns to uint32 (negative values
// reversed below the positive ones), so that every pattern has a place.
__device__ __forceinline__ uint32_t x_order_key(float x)
{
    const uint32_t b = __float_as_uint(x);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__global__ void k_mech_place(const float* __restrict__ soa, uint32_t stride, const uint32_t* __restrict__ keys,
                             const uint32_t* __restrict__ slots, const uint32_t* __restrict__ start, uint32_t n,
                             uint2* __restrict__ placed)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const float x = soa[static_cast<size_t>(F_POS_X) * stride + g];
    placed[start[keys[g]] + slots[g]] = make_uint2(x_order_key(x), g);
}

template <bool SORDER>
__global__ void k_mech_order(const float* __restrict__ soa, uint32_t stride, const uint32_t* __restrict__ keys,
                             const uint32_t* __restrict__ start, const uint2* __restrict__ placed, uint32_t n,
                             uint32_t* __restrict__ sorder, float4* __restrict__ spos, float4* __restrict__ sprm)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t key = keys[g];
    const uint32_t s0 = start[key], s1 = start[key + 1];
    const float x = soa[static_cast<size_t>(F_POS_X) * stride + g];
    const uint32_t xk = x_order_key(x);
    uint32_t pi = s0, px = s0;
    for (uint32_t q = s0; q < s1; ++q) {
        const uint2 o = placed[q];
        pi += o.y < g ? 1u : 0u;
        px += (o.x < xk || (o.x == xk && o.y < g)) ? 1u : 0u;
    }
    if (SORDER) sorder[pi] = g;
    spos[px] = make_float4(x, soa[static_cast<size_t>(F_POS_Y) * stride + g], soa[static_cast<size_t>(F_POS_Z) * stride + g],
                           soa[static_cast<size_t>(F_RADIUS) * stride + g]);
    // square roots of the (non-negative) strengths: the pair factors
    // sqrt(rep_i rep_j), sqrt(adh_i adh_j) become one product each; the
    // cell's index in place of relmax, which only its reciprocal serves
    const float relmax = soa[static_cast<size_t>(F_REL_MAX_ADH) * stride + g];
    sprm[px] = make_float4(sqrtf(soa[static_cast<size_t>(F_REPULSION) * stride + g]),
                           sqrtf(soa[static_cast<size_t>(F_ADHESION) * stride + g]), __uint_as_float(g), 1.0f / relmax);
}

// The stable order alone, from the same binning (k_mech_order's first rank).
__global__ void k_mech_stable_order(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ start,
                                    const uint2* __restrict__ placed, uint32_t n, uint32_t* __restrict__ sorder)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t key = keys[g];
    const uint32_t s0 = start[key], s1 = start[key + 1];
    uint32_t pi = s0;
    for (uint32_t q = s0; q < s1; ++q) pi += placed[q].y < g ? 1u : 0u;
    sorder[pi] = g;
}

__device__ __forceinline__ uint32_t nbr_hash(uint32_t j)
{
    uint32_t x = j + 0x9E3779B9u;
    x ^= x >> 16;
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    x *= 0xC2B2AE35u;
    x ^= x >> 16;
    return x;
}

// Distance from c to the mechanics-voxel slab [lo, lo + vs) along one axis,
// slabs at the grid edge reaching to infinity (clamped cells), minus a
// 0.01 um margin that covers FP32 rounding of positions and bounds.
__device__ __forceinline__ float slab_gap(float c, float lo, float vs, int idx, int nidx)
{
    const float l = idx == 0 ? -INFINITY : lo;
    const float h = idx == nidx - 1 ? INFINITY : lo + vs;
    return fmaxf(fmaxf(l - c, c - h) - 0.01f, 0.0f);
}

// One pair's force terms (mechanics.metal:167-208) added to the running
// sums: d = p_i - p_j with dsq = |d|^2 (the test's exact FP32 value), Ri /
// Rj the radii, mp = (sqrt rep_i, sqrt adh_i, -, 1 / relmax_i), op
// the strengths of j.  Reciprocal / rsqrt forms and per-cell square roots
// of the strengths (a few ulp per term against the reference's sqrt and
// divides); dist / (relmax_i R) is taken as (dist / R) / relmax_i.  Every
// product, sum and fused multiply-add is written out with its rounding, so
// the terms have the same bits in every kernel that inlines this, whatever
// the compiler would contract around it.
__device__ __forceinline__ void pair_force(float ddx, float ddy, float ddz, float dsq, float Ri, float Rj,
                                           const float4& mp, const float4& op, float& fx, float& fy, float& fz,
                                           float& P)
{
    constexpr float kInvPressureScale = 1.0f / 0.027288820670331f;
    const float inv = rsqrtf(dsq);
    const float dist = __fmul_rn(dsq, inv);
    const float u = __fdividef(dist, __fadd_rn(Ri, Rj));               // dist / R
    const float ov = fmaxf(__fsub_rn(1.0f, u), 0.0f);                   // repulsion overlap
    const float t = fmaxf(__fmaf_rn(-u, mp.w, 1.0f), 0.0f);             // adhesion reach
    const float ov2 = __fmul_rn(ov, ov);
    const float F = __fmaf_rn(ov2, __fmul_rn(mp.x, op.x), -__fmul_rn(__fmul_rn(t, t), __fmul_rn(mp.y, op.y)));
    P = __fmaf_rn(ov2, kInvPressureScale, P);
    const float Fi = __fmul_rn(F, inv);
    fx = __fmaf_rn(Fi, ddx, fx);
    fy = __fmaf_rn(Fi, ddy, fy);
    fz = __fmaf_rn(Fi, ddz, fz);
}

// One thread per cell, cells in the force order p (by mechanics voxel,
// then x; the cell's index is the bits of sprm[p].z).  Candidates are the cells of the 3 x 3 (x 3)
// voxels around the cell's own (mechanics.metal:125-208), visited row by
// row (dk, then dj), each row of three voxels along x being one run of the
// force order sorted by x.  A row whose slab lies beyond the interaction
// distance in y / z is skipped; in the others only the candidates whose x
// lies within sqrt(d^2 - g^2) (+ 0.05 um) of the cell's are tested, g the
// row's y / z gap: the walk skips the lower end of the row and stops at the
// first candidate past the upper bound.  Every candidate that can pass is
// tested, with the reference's FP32 test without contraction
// (mechanics.metal:159-165), so neighbour sets are exact (for finite
// positions).  The force terms follow pair_force.
//
// QCAP == 0: the walk takes two candidates a step, both positions and both
// strengths loaded before either is tested (four independent loads in
// flight per lane), and the force terms are computed where a lane meets its
// neighbour.  QCAP > 0: the walk only tests; each lane keeps the
// candidates that pass, in order, in its own QCAP slots of shared memory
// (slot k of thread t at queue[k * blockDim + t]; the next candidate's
// position is loaded while the current one is tested), and the force terms of
// the queued neighbours are computed when a lane's queue is full (every
// lane walking with it then empties its own) and at the end.  Every lane
// adds its terms in candidate order either way, so both forms give the same
// bits; the queued form runs the force terms for the neighbours only,
// where the direct form runs them whenever any lane of the warp has one.
// Registers are capped at 48 (five blocks of 256 threads per SM; part of
// the row table spills to L1): the walk is bound by load latency, and the
// extra resident warps hide more of it than the spills cost.
template <int QCAP, bool DIAG>
__global__ void __launch_bounds__(256, 5) k_mech_forces(const float4* __restrict__ spos, const float4* __restrict__ sprm,
                                                     const uint32_t* __restrict__ start, uint32_t n,
                                                     const uint32_t* __restrict__ cell_inst,
                                                     const CellInst* __restrict__ insts, float* __restrict__ soa,
                                                     uint32_t stride, uint32_t* __restrict__ diag_cnt,
                                                     uint32_t* __restrict__ diag_hash,
                                                     const uint8_t* __restrict__ mask)
{
    extern __shared__ uint32_t queue[];
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float4 mp = sprm[p];
    const uint32_t g = __float_as_uint(mp.z);
    const uint32_t ii = cell_inst[g];
    if (mask && !(mask[ii] & STEP_MECH)) return;
    const CellInst& in = insts[ii];
    const float4 me = spos[p];
    const int mnx = static_cast<int>(in.mnx), mny = static_cast<int>(in.mny), mnz = static_cast<int>(in.mnz);
    // the cell's voxel, from its position exactly as k_mech_bin binned it
    const int ci = clampi(bin_of(me.x, in.mx_min, in.vs), 0, mnx - 1);
    const int cj = clampi(bin_of(me.y, in.my_min, in.vs), 0, mny - 1);
    const int ck = clampi(bin_of(me.z, in.mz_min, in.vs), 0, mnz - 1);
    const float vs = in.vs;
    const float maxd2 = __fmul_rn(in.maxd, in.maxd);
    const int ilo = ci > 0 ? ci - 1 : 0, ihi = ci + 1 < mnx ? ci + 1 : mnx - 1;
    // row ranges [q0, q1) of the cell-start table, dk-major then dj, and
    // each row's half-width of the x window (negative: row skipped)
    uint32_t rq0[9], rq1[9];
    float rw[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        const int dk = r / 3 - 1, dj = r % 3 - 1;
        const int nk = ck + dk, nj = cj + dj;
        rq0[r] = rq1[r] = 0;
        rw[r] = -1.0f;
        if ((mnz == 1 && dk != 0) || nk < 0 || nk >= mnz || nj < 0 || nj >= mny) continue;
        const float gz = mnz > 1 ? slab_gap(me.z, in.mz_min + nk * vs, vs, nk, mnz) : 0.f;
        const float gy = slab_gap(me.y, in.my_min + nj * vs, vs, nj, mny);
        const float gyz = gy * gy + gz * gz;
        if (gyz >= maxd2) continue;   // the whole row is out of reach
        const uint32_t row = in.mvox_base + static_cast<uint32_t>(nk * mny + nj) * static_cast<uint32_t>(mnx);
        rq0[r] = start[row + ilo];
        rq1[r] = start[row + ihi + 1];
        rw[r] = __fsqrt_rn(maxd2 - gyz) + 0.05f;
    }
    float fx = 0.f, fy = 0.f, fz = 0.f, P = 0.f;
    uint32_t cnt = 0, hsh = 0;
    uint32_t* myq = queue + threadIdx.x;
    const uint32_t qstride = blockDim.x;
    uint32_t nq = 0;
    // force terms of the queued neighbours, in the order they were queued
    auto flush = [&]() {
        for (uint32_t k = 0; k < nq; ++k) {
            const uint32_t q = myq[k * qstride];
            const float4 cur = spos[q];
            const float ddx = __fsub_rn(me.x, cur.x), ddy = __fsub_rn(me.y, cur.y), ddz = __fsub_rn(me.z, cur.z);
            const float dsq = __fadd_rn(__fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy)), __fmul_rn(ddz, ddz));
            pair_force(ddx, ddy, ddz, dsq, me.w, cur.w, mp, sprm[q], fx, fy, fz, P);
        }
        nq = 0;
    };
    const float* sx = reinterpret_cast<const float*>(spos);   // x of position q at sx[4 q]
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        uint32_t q = rq0[r];
        const uint32_t q1 = rq1[r];
        const float xlo = me.x - rw[r], xhi = me.x + rw[r];
        // first candidate above the window's lower bound: a binary search
        // over the row, the same number of steps for every lane
        for (uint32_t len = q1 - q; len > 0;) {
            const uint32_t half = len >> 1;
            if (sx[4 * (q + half)] <= xlo) {
                q += half + 1;
                len -= half + 1;
            } else {
                len = half;
            }
        }
        if (QCAP == 0) {
            // two candidates a step, positions and strengths of both loaded
            // before either is tested (q + 1 <= q1 <= n: spos and sprm have
            // one spare element)
            while (q < q1) {
                const float4 c0 = spos[q], c1 = spos[q + 1];
                const float4 p0 = sprm[q], p1 = sprm[q + 1];
                bool more = true;
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const float4& cur = k == 0 ? c0 : c1;
                    // past the row or the window: so is every later candidate of the row
                    const bool in_win = q + k < q1 && cur.x < xhi;
                    if (in_win) {
                        // neighbour test exactly as mechanics.metal:159-165 (no contraction);
                        // the cell itself (distance 0) fails it like any coincident cell
                        const float ddx = __fsub_rn(me.x, cur.x), ddy = __fsub_rn(me.y, cur.y),
                                    ddz = __fsub_rn(me.z, cur.z);
                        const float dsq =
                            __fadd_rn(__fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy)), __fmul_rn(ddz, ddz));
                        if (!(dsq >= maxd2 || dsq < 1e-12f)) {
                            if (DIAG) {
                                ++cnt;
                                hsh += nbr_hash(__float_as_uint((k == 0 ? p0 : p1).z) - in.cell_off);
                            }
                            pair_force(ddx, ddy, ddz, dsq, me.w, cur.w, mp, k == 0 ? p0 : p1, fx, fy, fz, P);
                        }
                    }
                    more = in_win;
                }
                if (!more) break;
                q += 2;
            }
            continue;
        }
        float4 o = spos[q];   // q <= n: in bounds even for an empty row
        for (; q < q1; ++q) {
            const float4 cur = o;
            o = spos[q + 1];   // next candidate in flight (spos has one spare element)
            if (cur.x >= xhi) break;   // this and every later candidate of the row lie past the window
            // neighbour test exactly as mechanics.metal:159-165 (no contraction)
            const float ddx = __fsub_rn(me.x, cur.x), ddy = __fsub_rn(me.y, cur.y), ddz = __fsub_rn(me.z, cur.z);
            const float dsq = __fadd_rn(__fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy)), __fmul_rn(ddz, ddz));
            const bool nb = !(dsq >= maxd2 || dsq < 1e-12f);
            if (DIAG && nb) {
                ++cnt;
                hsh += nbr_hash(__float_as_uint(sprm[q].z) - in.cell_off);
            }
            if (nb) myq[nq++ * qstride] = q;
            if (__any_sync(__activemask(), nq == QCAP)) flush();
        }
    }
    if (QCAP > 0) flush();
    soa[static_cast<size_t>(F_VEL_X) * stride + g] = fx;
    soa[static_cast<size_t>(F_VEL_Y) * stride + g] = fy;
    soa[static_cast<size_t>(F_VEL_Z) * stride + g] = fz;
    soa[static_cast<size_t>(F_PRESSURE) * stride + g] = P;
    if (DIAG) {
        diag_cnt[g] = cnt;
        diag_hash[g] = hsh;
    }
}

// AB2 in FP64 with explicit rounding (integrate.metal:58-69 forms
// p + dt (1.5 v - 0.5 v_prev) and clamps it to the box of the mechanics
// grid): the FP64 value is clamped, kept as the cell's master position and
// rounded once into the FP32 SoA.  The update starts from the master while
// it rounds to the SoA's FP32 value, else (no master yet, or the FP32
// position was written since) from the FP32 value.
__global__ void k_mech_integrate(float* __restrict__ soa, double* __restrict__ pos64, uint32_t stride, uint32_t n,
                                 const uint32_t* __restrict__ cell_inst, const CellInst* __restrict__ insts,
                                 float dt_override, const uint8_t* __restrict__ mask)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t ii = cell_inst[g];
    if (mask && !(mask[ii] & STEP_MECH)) return;
    const CellInst& in = insts[ii];
    const double dt = static_cast<double>(dt_override >= 0.0f ? dt_override : in.dt_mech);
    const float lo[3] = {in.mx_min, in.my_min, in.mz_min};
    const float hi[3] = {in.box_hi_x, in.box_hi_y, in.box_hi_z};
    float pos[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float* p = soa + static_cast<size_t>(F_POS_X + a) * stride + g;
        const float v = soa[static_cast<size_t>(F_VEL_X + a) * stride + g];
        float* pv = soa + static_cast<size_t>(F_PREV_VX + a) * stride + g;
        const float p32 = *p;
        double x0 = static_cast<double>(p32);
        if (pos64) {
            const double m = pos64[static_cast<size_t>(a) * stride + g];
            if (__double2float_rn(m) == p32) x0 = m;
        }
        const double inc = __dsub_rn(__dmul_rn(1.5, static_cast<double>(v)), __dmul_rn(0.5, static_cast<double>(*pv)));
        double x = __dadd_rn(x0, __dmul_rn(dt, inc));
        if (x < static_cast<double>(lo[a])) x = lo[a];
        if (x > static_cast<double>(hi[a])) x = hi[a];
        if (pos64) pos64[static_cast<size_t>(a) * stride + g] = x;
        pos[a] = __double2float_rn(x);
        *p = pos[a];
        *pv = v;
    }
    if (in.flags & INST_REFRESH_VOXELS) {
        const int i = clampi(bin_of(pos[0], in.x_min, in.dx), 0, static_cast<int>(in.nx) - 1);
        const int j = clampi(bin_of(pos[1], in.y_min, in.dy), 0, static_cast<int>(in.ny) - 1);
        const int k = clampi(bin_of(pos[2], in.z_min, in.dz), 0, static_cast<int>(in.nz) - 1);
        const uint32_t v = static_cast<uint32_t>(k) * in.nx * in.ny + static_cast<uint32_t>(j) * in.nx +
                           static_cast<uint32_t>(i);
        soa[static_cast<size_t>(F_VOXEL_IDX) * stride + g] = __uint_as_float(v);
    }
}

// ------------------------------------------------------------------ launchers

static inline unsigned blocks_for(uint64_t n, int b) { return static_cast<unsigned>((n + b - 1) / b); }

cudaError_t launch_sec_cell_consts(cudaStream_t st, const float* soa, uint32_t stride, uint32_t n,
                                   const uint32_t* cell_inst, const CellInst* insts, const double* rates4,
                                   uint32_t n_rate, double dt, double* cc, uint32_t* flags, uint32_t n_inst)
{
    cudaError_t e = cudaMemsetAsync(flags, 0, static_cast<size_t>(n_inst) * sizeof(uint32_t), st);
    if (e != cudaSuccess || n == 0) return e;
    k_sec_cell_consts<<<blocks_for(n, 256), 256, 0, st>>>(soa, stride, n, cell_inst, insts, rates4, n_rate, dt, cc,
                                                           flags);
    return cudaGetLastError();
}

cudaError_t launch_sec_permute(cudaStream_t st, const uint32_t* skeys, const uint32_t* sorder, uint32_t n,
                               const uint32_t* cell_inst, const CellInst* insts, uint32_t invalid_key,
                               const uint32_t* flags, const double* cc, uint32_t n_rate, double* cs)
{
    if (n == 0) return cudaSuccess;
    k_sec_permute<<<blocks_for(n, 256), 256, 0, st>>>(skeys, sorder, n, cell_inst, insts, invalid_key, flags, cc,
                                                       n_rate, cs);
    return cudaGetLastError();
}

cudaError_t launch_secrete(cudaStream_t st, float* dens, const uint32_t* run_start, const uint64_t* run_word,
                           const uint32_t* n_runs, uint32_t max_runs, uint32_t max_s, const CellInst* insts, const double* cs, uint32_t cap,
                           const uint32_t* flags, const uint8_t* mask, int block)
{
    if (max_runs == 0 || max_s == 0) return cudaSuccess;
    if (block < 32 || block > 256 || block % 32) return cudaErrorInvalidValue;
    k_secrete<<<blocks_for(max_runs, block), block, 0, st>>>(dens, run_start, run_word, n_runs, insts, cs, cap, flags,
                                                          mask);
    return cudaGetLastError();
}

cudaError_t launch_cells_move(cudaStream_t st, float* soa, uint32_t stride, const uint2* moves, uint32_t n_moves,
                              double* rates, uint64_t rate_cap, uint32_t S, uint8_t* active, double* pos64)
{
    const uint64_t work = static_cast<uint64_t>(n_moves) * (NUM_FIELDS + 4u * S + 1u + 3u);
    if (work == 0) return cudaSuccess;
    k_cells_move<<<blocks_for(work, 256), 256, 0, st>>>(reinterpret_cast<uint32_t*>(soa), stride, moves, n_moves, rates,
                                                       rate_cap, S, active, pos64);
    return cudaGetLastError();
}

cudaError_t launch_mech_bin(cudaStream_t st, float* soa, uint32_t stride, uint32_t n, const uint32_t* cell_inst,
                            const CellInst* insts, uint32_t* keys, uint32_t* slots, uint32_t* counts,
                            const uint8_t* mask, int block)
{
    if (n == 0) return cudaSuccess;
    if (block < 32 || block > 1024 || block % 32) return cudaErrorInvalidValue;
    k_mech_bin<<<blocks_for(n, block), block, 0, st>>>(soa, stride, n, cell_inst, insts, keys, slots, counts, mask);
    return cudaGetLastError();
}

cudaError_t launch_mech_order(cudaStream_t st, const float* soa, uint32_t stride, const uint32_t* keys,
                              const uint32_t* slots, const uint32_t* start, uint32_t n, uint2* placed,
                              uint32_t* sorder, float4* spos, float4* sprm, int block)
{
    if (n == 0) return cudaSuccess;
    if (block < 32 || block > 1024 || block % 32) return cudaErrorInvalidValue;
    k_mech_place<<<blocks_for(n, block), block, 0, st>>>(soa, stride, keys, slots, start, n, placed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (sorder)
        k_mech_order<true><<<blocks_for(n, block), block, 0, st>>>(soa, stride, keys, start, placed, n, sorder, spos,
                                                                   sprm);
    else
        k_mech_order<false><<<blocks_for(n, block), block, 0, st>>>(soa, stride, keys, start, placed, n, nullptr, spos,
                                                                    sprm);
    return cudaGetLastError();
}

cudaError_t launch_mech_stable_order(cudaStream_t st, const uint32_t* keys, const uint32_t* start,
                                     const uint2* placed, uint32_t n, uint32_t* sorder)
{
    if (n == 0) return cudaSuccess;
    k_mech_stable_order<<<blocks_for(n, 256), 256, 0, st>>>(keys, start, placed, n, sorder);
    return cudaGetLastError();
}

template <int QCAP, bool DIAG>
static cudaError_t forces_variant(cudaStream_t st, unsigned grid, int block, const float4* spos, const float4* sprm,
                                  const uint32_t* start, uint32_t n,
                                  const uint32_t* cell_inst, const CellInst* insts, float* soa, uint32_t stride,
                                  uint32_t* diag_cnt, uint32_t* diag_hash, const uint8_t* mask)
{
    const size_t smem = static_cast<size_t>(QCAP) * block * sizeof(uint32_t);   // at most 64 KiB
    k_mech_forces<QCAP, DIAG><<<grid, block, smem, st>>>(spos, sprm, start, n, cell_inst, insts, soa, stride,
                                                         diag_cnt, diag_hash, mask);
    return cudaGetLastError();
}

cudaError_t mech_forces_prepare()
{
    const void* ks[] = {reinterpret_cast<const void*>(&k_mech_forces<64, false>),
                        reinterpret_cast<const void*>(&k_mech_forces<64, true>)};
    for (const void* k : ks) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_mech_forces(cudaStream_t st, const float4* spos, const float4* sprm,
                               const uint32_t* start, uint32_t n, const uint32_t* cell_inst,
                               const CellInst* insts, float* soa, uint32_t stride, uint32_t* diag_cnt,
                               uint32_t* diag_hash, const uint8_t* mask, ForceShape shape)
{
    if (n == 0) return cudaSuccess;
    if (shape.block < 32 || shape.block > 256 || shape.block % 32 != 0) return cudaErrorInvalidValue;
    const unsigned grid = blocks_for(n, shape.block);
    const bool dg = diag_cnt != nullptr;
#define PCG_FORCES(Q)                                                                                                \
    return dg ? forces_variant<Q, true>(st, grid, shape.block, spos, sprm, start, n, cell_inst, insts, soa, stride, \
                                        diag_cnt, diag_hash, mask)                                                   \
              : forces_variant<Q, false>(st, grid, shape.block, spos, sprm, start, n, cell_inst, insts, soa, stride, \
                                         diag_cnt, diag_hash, mask)
    switch (shape.queue) {
    case 0: PCG_FORCES(0);
    case 16: PCG_FORCES(16);
    case 32: PCG_FORCES(32);
    case 64: PCG_FORCES(64);
    default: return cudaErrorInvalidValue;
    }
#undef PCG_FORCES
}

cudaError_t launch_mech_integrate(cudaStream_t st, float* soa, double* pos64, uint32_t stride, uint32_t n,
                                  const uint32_t* cell_inst, const CellInst* insts, float dt_override,
                                  const uint8_t* mask, int block)
{
    if (n == 0) return cudaSuccess;
    if (block < 32 || block > 1024 || block % 32) return cudaErrorInvalidValue;
    k_mech_integrate<<<blocks_for(n, block), block, 0, st>>>(soa, pos64, stride, n, cell_inst, insts, dt_override,
                                                             mask);
    return cudaGetLastError();
}

uint32_t neighbor_hash_host(uint32_t j)
{
    uint32_t x = j + 0x9E3779B9u;
    x ^= x >> 16;
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    x *= 0xC2B2AE35u;
    x ^= x >> 16;
    return x;
}

}  // namespace pcg
