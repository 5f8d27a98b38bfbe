// pcg_kernels.cuh — device data structures shared by the sm_100a kernels and
// the host runtime, and the host-side launchers of every kernel.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace pcg {

// Cell SoA field ids (shaders/types.h:74-102).
enum Field : int {
    F_POS_X = 0, F_POS_Y = 1, F_POS_Z = 2,
    F_VEL_X = 3, F_VEL_Y = 4, F_VEL_Z = 5,
    F_PREV_VX = 6, F_PREV_VY = 7, F_PREV_VZ = 8,
    F_RADIUS = 9, F_TOTAL_VOL = 11,
    F_REPULSION = 13, F_ADHESION = 14, F_REL_MAX_ADH = 15, F_MOT_SPEED = 16,
    F_PRESSURE = 22, F_IS_ALIVE = 25, F_VOXEL_IDX = 26, F_MECH_VOXEL = 27,
    NUM_FIELDS = 28
};

// ---------------------------------------------------------------- diffusion

// Thomas constants of one (instance, substrate, axis) line family.  Every
// line of the family has the same matrix, so g_i = c / den_i and
// inv_i = 1 / den_i are one table built on the host in FP64 from the
// reference's recurrence (shaders/diffusion_2d.metal:86-148):
//   forward   d_1 = (rho_1 + fold) / b_bnd
//             d_i = (rho_i [+ fold at i = n-2] + c d_{i-1}) / den_i
//   backward  rho_i = d_i - c'_i rho_{i+1}
// with den_i = b + c c'_{i-1}, c'_i = -c / den_i = -g_i; written as
// d_i = fma(g_i, d_{i-1}, (rho_i + fold_i) * inv_i), x_i = fma(g_i, x_{i+1}, d_i).
// Table layout: line positions in chunks of 4, chunk q at tab + 8 q holds
// {g[4q..4q+3], inv[4q..4q+3]} (32-byte aligned; zero at the end nodes).
struct LineRule {
    uint32_t tab;   // first float of the rule's table (multiple of 8)
    uint32_t n;     // line length
    float c;        // D dt / h^2
    float fold;     // Dirichlet RHS fold: c T (2 c T when n == 3), 0 without Dirichlet
    float T;        // Dirichlet target
    uint32_t dir;   // Dirichlet enabled
    uint32_t inst;  // instance index (step mask lookup)
    uint32_t _pad;
};

// Floats of table for a line of n positions.
__host__ __device__ constexpr uint32_t tab_floats(uint32_t n) { return ((n + 3u) / 4u) * 8u; }

// A tile of lines for one sweep launch.  Row tiles (x sweep, TILE_ROWS):
// 'count' (<= 32) lines of length n starting at element 'base', lines 'rs'
// (the row pitch) apart.  Column tiles (y and z sweeps): 'nslab' adjacent
// slabs (outer coordinates outer .. outer + nslab - 1) of 'count' (<= width)
// adjacent columns from x = i0, width * nslab <= 32; lane = slab * width +
// column.  Without a tensor map a column tile has width 32 and one slab, and
// its lines start at 'base' with element stride 'rs'.
struct SweepTile {
    uint64_t base;
    uint32_t count;
    uint32_t rs;       // row tiles: line pitch; column tiles: element stride along a line
    uint32_t i0;       // x index of the tile's first column (column tiles)
    uint32_t nx;       // the instance's nx
    uint32_t face;     // TILE_FACE: the Dirichlet reset is fused into this sweep;
                       // TILE_ROWS: x tile; TILE_TENSOR: moved with tensor map 'map';
                       // TILE_AXIS_Z: z tile (else y)
    uint32_t outer;    // column tiles: first slab (k for y, j for z); row tiles: first line
    uint32_t map;      // index of the 128-byte tensor map
    uint16_t width;    // columns per slab (column tiles): 32, 16 or 8
    uint16_t nslab;    // slabs in the tile
    uint32_t outer_n;  // number of slabs (nz for y, ny for z)
    // the tile's line rule (LineRule), carried in the descriptor so that a
    // tile costs one descriptor load
    uint32_t n;        // line length
    uint32_t tab;      // first float of the coefficient table
    float fold;        // Dirichlet RHS fold
    float T;           // Dirichlet target
    uint32_t inst;     // instance index; bit 31 set: Dirichlet
};
static_assert(sizeof(SweepTile) == 64, "one 64-byte descriptor per tile");
enum : uint32_t { TILE_FACE = 1u, TILE_ROWS = 4u, TILE_TENSOR = 8u, TILE_AXIS_Z = 16u };

// Longest line a tensor-map box can cover (box dimensions are <= 256).
constexpr uint32_t kTensorMaxN = 256;
// Tensor-map slots per rule: x rules use slot 0, y / z rules one per
// column-tile width (32, 16, 8).
constexpr uint32_t kMapsPerRule = 4;

// x tiles moved with a 2-D tensor map land in shared memory as 32 rows of
// row_smem_pitch(nx) floats: nx rounded up to 4 with an odd number of
// 16-byte groups, so 16-byte accesses of the 32 rows are free of bank
// conflicts.  The box must fit 256 floats.
__host__ __device__ constexpr uint32_t row_smem_pitch(uint32_t n) { return (((n + 3u) / 4u) | 1u) * 4u; }
constexpr uint32_t kRowTensorMaxN = 252;

// Device status word bits (a kernel that cannot finish records why and returns).
enum : unsigned { PCG_DEV_TIMEOUT = 1u, PCG_DEV_ALIGN = 2u };
// Test switches, in the word after the status word: PCG_DEV_TEST_GIVE_UP
// makes the first wait of every plane CTA report that its bound ran out at
// once (the wait for the CTA's own copies before it exits keeps its bound).
enum : unsigned { PCG_DEV_TEST_GIVE_UP = 1u };

// ---------------------------------------------------------------- cells

// Per-instance constants for secretion, binning, forces and integration.
struct CellInst {
    // diffusion grid (secretion, voxel refresh)
    uint32_t nx, ny, nz, S;
    float dx, dy, dz;
    uint32_t flags;        // INST_REFRESH_VOXELS
    float x_min, y_min, z_min, dt_mech;
    uint64_t dens_off;     // element offset of substrate 0 in the density arena
    uint64_t sub_pitch;    // elements between substrates
    uint32_t px;           // row pitch (floats) of the density layout
    uint32_t _pad_px;
    uint32_t vox_base;     // global diffusion-voxel key of voxel 0
    uint32_t cell_off;     // global index of the instance's first cell
    uint32_t n_cells;
    uint32_t rate_off;     // index of (cell 0, substrate 0) in the rate arrays
    // mechanics grid (cell_mechanics.mm:26-70): origin, voxel, clamp box
    uint32_t mnx, mny, mnz, mvox_base;
    float vs, maxd, mx_min, my_min;
    float mz_min, box_hi_x, box_hi_y, box_hi_z;
};

enum : uint32_t { INST_REFRESH_VOXELS = 1u };

// Per-instance step mask (nullptr = every instance runs): bit 0 = the
// instance takes this diffusion step, bit 1 = it takes this mechanics step.
enum : uint8_t { STEP_DIFFUSE = 1u, STEP_MECH = 2u };

// ---------------------------------------------------------------- launchers
// All launchers enqueue on 'st' and return the CUDA launch status.

// Pipelined TMA sweeps: 'warps' warps per CTA, each with 'stages' shared
// memory stages of 'stage_floats' floats, the last 'tab_floats' of which
// hold the tile's coefficient table; 'grid' persistent CTAs.
// One plane for the plane sweep kernel, of width nx (columns) and height ny
// (rows).  x-y jobs (z slab k of one instance-substrate): the plane tensor
// map (box row_smem_pitch(nx) x ny, slot 1 of the x rule), first row
// row0 = k * ny, x and y rules: every row, then every column is solved.
// z jobs (kPlaneZ: the x-z plane y = row0): the 3-D map of slot 3 of the z
// rule (box round4(nx) x 1 x nz), ny = nz, the z rule in the y fields:
// every column (a z line) is solved.
struct PlaneJob {
    uint32_t map;
    uint32_t row0;
    uint32_t nx, ny;
    uint32_t tab_x, tab_y;   // table offsets (floats)
    float fold_x, T_x, fold_y, T_y;
    uint32_t inst;           // instance | kPlaneDirX | kPlaneDirY | kPlaneFaces | kPlaneZ | kPlaneSlabFace
    uint32_t _pad[5];
};
static_assert(sizeof(PlaneJob) == 64, "PlaneJob is 64 bytes");
constexpr uint32_t kPlaneDirX = 1u << 31, kPlaneDirY = 1u << 30, kPlaneFaces = 1u << 29;
constexpr uint32_t kPlaneZ = 1u << 28;          // an x-z plane of z lines
constexpr uint32_t kPlaneSlabFace = 1u << 27;   // z job: the plane is a y face of the block
constexpr uint32_t kPlaneInstMask = (1u << 27) - 1u;
constexpr uint32_t kPlaneThreads = 128;
// Row pitch of a plane in shared memory: x-y planes row_smem_pitch(nx) (the
// rows are solved with 16-byte accesses), z planes nx rounded up to 4.
__host__ __device__ constexpr uint32_t plane_pitch(uint32_t nx, bool z)
{
    return z ? ((nx + 3u) & ~3u) : row_smem_pitch(nx);
}
// Shared floats of a plane's data (rows rounded up to a whole chunk of 4,
// which the column solve may touch; 128-byte multiple) and with its tables.
__host__ __device__ constexpr uint32_t plane_data_floats(uint32_t nx, uint32_t ny, bool z = false)
{
    return (plane_pitch(nx, z) * ((ny + 3u) & ~3u) + 31u) / 32u * 32u;
}
__host__ __device__ constexpr uint32_t plane_floats(uint32_t nx, uint32_t ny, bool z = false)
{
    return plane_data_floats(nx, ny, z) + (z ? 0u : tab_floats(nx)) + tab_floats(ny);
}

struct TmaCfg { int warps; int stages; int stage_floats; int grid; int tab_floats; };

// Longest line staged in shared memory; longer lines take the one-thread-
// per-line kernel.  Tables are the chunked LineRule tables (float).
constexpr uint32_t kTmaMaxN = 512;

size_t sweep_tma_smem(int warps, int nstages, int stage_floats);
int sweep_tma_occupancy(bool rows, int warps, int nstages, int stage_floats);   // CTAs per SM (0 = does not fit)
// tmaps: one 128-byte CUtensorMap per rule (64-byte aligned, global memory)
// for the tiles flagged TILE_TENSOR; may be null otherwise.
// Fused x + y sweeps, one CTA per plane; 'floats' = the largest
// plane_floats of the jobs.
cudaError_t launch_sweep_planes(cudaStream_t st, const PlaneJob* jobs, uint32_t njobs, const float* tab,
                                const void* tmaps, uint32_t floats, int apply_faces, const uint8_t* mask,
                                unsigned* status);
// Lets the plane kernel use the opt-in shared memory, with the largest
// shared-memory carveout, so launches of every plane size share one SM
// configuration (current device; once per device, outside stream capture).
cudaError_t sweep_planes_prepare();
size_t sweep_planes_smem(uint32_t floats);
// Plane CTAs an SM holds at once for planes of 'floats' (0 = does not fit);
// sweep_planes_prepare() first.
int sweep_planes_ctas(uint32_t floats);
bool encode_plane_map(void* map128, float* block, uint32_t nx, uint32_t ny, uint64_t rows, uint32_t px);
bool encode_xz_plane_map(void* map128, float* block, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t px);
cudaError_t launch_sweep_tma(cudaStream_t st, bool rows, float* dens, const SweepTile* tiles, uint32_t ntiles,
                             const float* tab, const void* tmaps, int apply_faces,
                             const uint8_t* mask, unsigned* status, TmaCfg cfg);
// Encode the 3-D tensor map of one substrate block (rows px floats apart)
// for column tiles of 'width' columns x 32/width slabs x n line positions:
// y sweep dims (x, z, y), z sweep dims (x, y, z), box {width, 32/width, n},
// so a tile lands in shared memory as [n][32].  Returns false when the
// driver entry point is unavailable or rejects the map.
bool encode_column_map(void* map128, float* block, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t px, int axis,
                       uint32_t n, uint32_t width);
// Encode the 2-D tensor map of one substrate block seen as rows x nx (rows
// px floats apart) with a box of row_smem_pitch(nx) x 32 (x tiles).
bool encode_row_map(void* map128, float* block, uint32_t nx, uint64_t rows, uint32_t px);
// Any line length: one thread per line, d kept in place in global memory.
cudaError_t launch_sweep_global(cudaStream_t st, float* dens, const SweepTile* tiles, uint32_t ntiles,
                                const float* tab, int apply_faces, const uint8_t* mask,
                                int grid);

// applyDirichletBC over instances [0, n_inst): faces of Dirichlet substrates.
struct FaceJob { uint64_t base; uint32_t nx, ny, nz, px; float T; uint32_t _pad; };
cudaError_t launch_dirichlet(cudaStream_t st, float* dens, const FaceJob* jobs, uint32_t njobs);

// Central / one-sided gradients (microenvironment.mm:197-257).
struct GradJob { uint64_t base; uint64_t out_base; uint32_t nx, ny, nz, px; float inv_dx, inv_dy, inv_dz, _pad; };
cudaError_t launch_gradients(cudaStream_t st, const float* dens, float* gx, float* gy, float* gz,
                             const GradJob* jobs, uint32_t njobs, uint64_t max_voxels);

// Secretion: the order and its run list (launch_sec_order, below), the
// constants in cell order (cc: three arrays of n_rate doubles, c0, c1, c2)
// with the per-instance flags, their permutation into the order's slots
// (cs; c0 / c1 only for instances whose flags have them) and the ordered
// application.
cudaError_t launch_sec_cell_consts(cudaStream_t st, const float* soa, uint32_t stride, uint32_t n,
                                   const uint32_t* cell_inst, const CellInst* insts, const double* rates4,
                                   uint32_t n_rate, double dt, double* cc, uint32_t* flags, uint32_t n_inst);
cudaError_t launch_sec_permute(cudaStream_t st, const uint32_t* skeys, const uint32_t* sorder, uint32_t n,
                               const uint32_t* cell_inst, const CellInst* insts, uint32_t invalid_key,
                               const uint32_t* flags, const double* cc, uint32_t n_rate, double* cs);
// n_runs: device count (heads_rid[n]); max_runs >= it; max_s = largest S;
// runs whose word names kRunNone are skipped.
// cs: constants c0, c1, c2 as three arrays of cap; flags: per instance, bit 0
// some c0 not +0, bit 1 some c1 not +0 (written by launch_sec_cell_consts).
cudaError_t launch_secrete(cudaStream_t st, float* dens, const uint32_t* run_start, const uint64_t* run_word,
                           const uint32_t* n_runs,
                           uint32_t max_runs, uint32_t max_s, const CellInst* insts, const double* cs, uint32_t cap,
                           const uint32_t* flags, const uint8_t* mask, int block = 256);

// Mechanics binning as a counting sort: launch_mech_bin writes each cell's
// global mechanics-voxel key, counts it (counts: V + 1 zeroed words) and
// records its arrival slot; after the exclusive scan of the counts into
// start, launch_mech_order (two launches; placed: n scratch pairs) writes
// the stable order (sorder: cells by voxel, ascending index within a voxel;
// skipped when null) and, in the force order (by voxel, then x, index
// breaking ties), the positions / radii (spos) and the strengths (sprm:
// sqrt repulsion, sqrt adhesion, the cell's index as bits, 1 / relmax).
// launch_mech_stable_order writes sorder alone from the same binning.
cudaError_t launch_mech_bin(cudaStream_t st, float* soa, uint32_t stride, uint32_t n,
                            const uint32_t* cell_inst, const CellInst* insts,
                            uint32_t* keys, uint32_t* slots, uint32_t* counts, const uint8_t* mask, int block = 256);
cudaError_t launch_mech_order(cudaStream_t st, const float* soa, uint32_t stride, const uint32_t* keys,
                              const uint32_t* slots, const uint32_t* start, uint32_t n, uint2* placed,
                              uint32_t* sorder, float4* spos, float4* sprm, int block = 256);
cudaError_t launch_mech_stable_order(cudaStream_t st, const uint32_t* keys, const uint32_t* start,
                                     const uint2* placed, uint32_t n, uint32_t* sorder);
// Launch shape of the force pass: threads per block (a multiple of 32, at
// most 256) and the neighbour queue per thread (0 = force terms in the walk;
// 16, 32 or 64 slots of shared memory).  Every shape gives the same bits.
// The default is the shape the tuner chooses on the batched 3-D workload.
struct ForceShape {
    int block = 128;
    int queue = 0;
};
// Lets the 64-slot queue variants use 64 KiB of shared memory (current
// device; once per device, outside stream capture).
cudaError_t mech_forces_prepare();
cudaError_t launch_mech_forces(cudaStream_t st, const float4* spos, const float4* sprm,
                               const uint32_t* start, uint32_t n,
                               const uint32_t* cell_inst, const CellInst* insts, float* soa, uint32_t stride,
                               uint32_t* diag_cnt, uint32_t* diag_hash, const uint8_t* mask, ForceShape shape);
// Copies of a removal plan: (dst, src) pairs, each cell's 28 SoA fields,
// 4 x S rates (arrays of rate_cap doubles, [cell * S + s]), active flag and
// three FP64 master positions (arrays of stride doubles; pos64 may be null).
cudaError_t launch_cells_move(cudaStream_t st, float* soa, uint32_t stride, const uint2* moves, uint32_t n_moves,
                              double* rates, uint64_t rate_cap, uint32_t S, uint8_t* active, double* pos64);
// dt_override >= 0 replaces every instance's dt_mech.  pos64: FP64 master
// positions (three arrays of stride doubles) or null for FP32 positions.
cudaError_t launch_mech_integrate(cudaStream_t st, float* soa, double* pos64, uint32_t stride, uint32_t n,
                                  const uint32_t* cell_inst, const CellInst* insts, float dt_override,
                                  const uint8_t* mask, int block = 256);

// The secretion order (secorder.cu): every instance's cells sorted by
// (voxel index in the instance's grid, cell index), non-secreting cells
// (inactive, voxel index outside the grid, no substrates) after them; each
// instance keeps its range [cell_off, cell_off + n_cells).  A tile is up to
// 2048 consecutive cells of one instance: first cell, count, instance, the
// instance's first tile and its number of tiles.
struct SegTile {
    uint32_t first, count, inst, tb, nt;
    uint32_t _pad[3];
};
// A run's word: its instance in the top 24 bits, the density element of its
// voxel (substrate 0) in the low 40 (the rate slot of its first cell
// follows from its start and the instance: rate_off + (start - cell_off) *
// S).  kRunNone in the instance bits: the instance's non-secreting cells.
constexpr int kRunDensBits = 40;
constexpr uint64_t kRunDensMask = (uint64_t{1} << kRunDensBits) - 1u;
constexpr uint32_t kRunNone = 0xFFFFFFu;   // also the bound on instances per batch
__host__ __device__ __forceinline__ uint64_t make_run_word(uint32_t inst, uint64_t dens_elem)
{
    return (static_cast<uint64_t>(inst) << kRunDensBits) | dens_elem;
}
// Passes and digit bits for grids of at most max_local_voxels voxels.
void so_plan(uint32_t max_local_voxels, int* passes, int* digit_bits);
// Most tiles a store of max_cells cells over n_inst instances can need.
uint32_t so_max_tiles(uint32_t max_cells, uint32_t n_inst);
// The tiles of the instances' cell ranges (host, from the CellInst table),
// and the first tile of every instance that has cells.
void so_tiles(const CellInst* inst, uint32_t n_inst, std::vector<SegTile>& out, std::vector<uint32_t>& inst_tile);
size_t so_scratch_bytes(uint32_t max_tiles);
int so_launches(uint32_t ntiles, int passes, uint32_t n);
size_t so_run_scratch_bytes(uint32_t max_cells);
// Keys, the sort and the run list in one call.  Outputs: skeys (global
// voxel key vox_base + index, or invalid_key) and sorder (cell) per sorted
// position; *n_runs; run_start (n + 1) and run_word per run.  keys, ktmp
// and vtmp are n-entry work arrays;
// scratch: so_scratch_bytes, run_scratch: so_run_scratch_bytes; inst_tile:
// the n_inst_tiled entries of so_tiles.  With cc non-null the last pass
// also permutes the constants (cc in cell order, three arrays of cap) into
// the order's slots (cs), as launch_sec_permute does.
cudaError_t launch_sec_order(cudaStream_t st, const SegTile* tiles, uint32_t ntiles, const uint32_t* inst_tile,
                             uint32_t n_inst_tiled, uint32_t n, int passes,
                             int digit_bits, const float* soa, uint32_t stride, const CellInst* insts,
                             const uint8_t* active, const uint32_t* cell_inst, uint32_t invalid_key, uint32_t* keys,
                             uint32_t* ktmp, uint32_t* vtmp, uint32_t* skeys, uint32_t* sorder, void* scratch,
                             uint32_t* n_runs, uint32_t* run_start, uint64_t* run_word, void* run_scratch,
                             const double* cc, double* cs, uint32_t cap, const uint32_t* flags);

// Radix sort of (key, value) pairs, stable, 'bits' significant key bits.
// Scratch from radix_sort_scratch_bytes().  Result lands in (k_out, v_out).
size_t radix_sort_scratch_bytes(uint32_t n, int bits);
int radix_sort_launches(uint32_t n, int bits);
cudaError_t radix_sort_pairs(cudaStream_t st, const uint32_t* k_in, const uint32_t* v_in,
                             uint32_t* k_out, uint32_t* v_out, uint32_t* k_tmp, uint32_t* v_tmp,
                             uint32_t n, int bits, void* scratch);

// Loads the radix sort's and the scan's kernels on the current device now
// rather than at their first launch.
cudaError_t sort_kernels_load();

// Exclusive prefix sum of n uint32 values (in may equal out).
size_t scan_scratch_bytes(uint64_t n);
int scan_launches(uint64_t n);
cudaError_t scan_exclusive(cudaStream_t st, const uint32_t* in, uint32_t* out, uint64_t n, void* scratch);

uint32_t neighbor_hash_host(uint32_t j);

}  // namespace pcg
