/*
 * pcg.h — C ABI of the B200 hot path of a PhysiCell-style simulator:
 * LOD Thomas diffusion-decay with Dirichlet boundaries and per-cell
 * secretion/uptake, spatial-hash cell-cell mechanics and the Adams-Bashforth
 * position update.
 *
 * Every entry point returns a pcg_status (PCG_OK == 0) and never aborts;
 * pcg_last_error_string() describes the last failure on a context.  Device
 * memory is owned by the library; host pointers stay owned by the caller.
 * Calls on one pcg_ctx are serialised on that context's CUDA stream and must
 * come from one host thread at a time; separate contexts may be used from
 * separate threads.  Floating-point layouts match the reference exactly:
 *   density   float32 [s][k][j][i]        (src/microenvironment.mm:48-60)
 *   cell SoA  float32 [field * max_cells + cell], 28 fields, fields 23..27
 *             hold uint32 bits            (src/cell_data.cpp:101-180,
 *                                          shaders/types.h:74-102)
 *   rates     float64 [cell * S + s]      (src/cell_data.cpp:380-394)
 */
#ifndef PCG_H
#define PCG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PCG_ABI_VERSION 1

typedef int pcg_status;
enum {
    PCG_OK = 0,
    PCG_ERR_INVALID = 1,     /* bad argument, size or state */
    PCG_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    PCG_ERR_OOM = 3,         /* device allocation failed */
    PCG_ERR_NO_DEVICE = 4,   /* no usable CUDA device */
    PCG_ERR_BUDGET = 5,      /* request does not fit the serving memory budget */
    PCG_ERR_NOT_FOUND = 6,   /* unknown request id */
    PCG_ERR_NOT_READY = 7,   /* request not finished yet */
    PCG_ERR_DEVICE = 8       /* a kernel stopped early (bounded wait ran out, unaligned copy refused) */
};

/* Same layout as GridParams (shaders/types.h:23-37). */
typedef struct {
    uint32_t nx, ny, nz, n_substrates;
    float dx, dy, dz, dt;
    float x_min, y_min, z_min, _pad0;
} pcg_grid_params;

/* Same layout as SubstrateParams (shaders/types.h:40-48); the first pad
 * word of the reference's struct holds an option the reference does not
 * have (0 there, the reference's behaviour):
 *   dirichlet_consistent != 0: on Dirichlet lines the first and last
 *   interior nodes use the interior diagonal 1 + 2c + hd rather than the
 *   reference's 1 + c + hd (diffusion_2d.metal:47-48, 90-142), keeping the
 *   c T coupling to the boundary value, so that a uniform field at the
 *   target stays there.  The reference's rule (both the boundary diagonal
 *   and the coupling) is the default, for parity. */
typedef struct {
    float diffusion_coefficient, decay_rate, supply_rate, target_value;
    uint32_t dirichlet_enabled;
    uint32_t dirichlet_consistent;
    float _pad[2];
} pcg_substrate_params;

/* Same layout as MechanicsParams (shaders/types.h:51-61). */
typedef struct {
    float dt, cell_cell_repulsion, cell_cell_adhesion, max_interaction_distance;
    float mechanics_voxel_size;
    uint32_t mech_grid_nx, mech_grid_ny, mech_grid_nz;
} pcg_mechanics_params;

/* Cell SoA field ids (shaders/types.h:74-102). */
enum {
    PCG_F_POS_X = 0, PCG_F_POS_Y, PCG_F_POS_Z,
    PCG_F_VEL_X, PCG_F_VEL_Y, PCG_F_VEL_Z,
    PCG_F_PREV_VX, PCG_F_PREV_VY, PCG_F_PREV_VZ,
    PCG_F_RADIUS, PCG_F_NUCLEAR_RAD, PCG_F_TOTAL_VOL, PCG_F_NUCLEAR_VOL,
    PCG_F_REPULSION, PCG_F_ADHESION, PCG_F_REL_MAX_ADH,
    PCG_F_MOT_SPEED, PCG_F_MOT_BIAS, PCG_F_MOT_DIR_X, PCG_F_MOT_DIR_Y, PCG_F_MOT_DIR_Z,
    PCG_F_ONCOPROTEIN, PCG_F_PRESSURE,
    PCG_F_CELL_TYPE, PCG_F_CUR_PHASE, PCG_F_IS_ALIVE, PCG_F_VOXEL_IDX, PCG_F_MECH_VOXEL,
    PCG_NUM_FIELDS
};

typedef struct pcg_ctx pcg_ctx;
typedef struct pcg_me pcg_me;
typedef struct pcg_cells pcg_cells;
typedef struct pcg_mech pcg_mech;
typedef struct pcg_motility pcg_motility;
typedef struct pcg_snapshot pcg_snapshot;
typedef struct pcg_batch pcg_batch;
typedef struct pcg_server pcg_server;

/* ------------------------------------------------------------------------
 * Context — replaces MetalContext (src/metal_context.h:14-100): device,
 * command queue (here a CUDA stream) and error reporting.
 * ---------------------------------------------------------------------- */
int pcg_abi_version(void);
pcg_status pcg_create(int device, pcg_ctx** out);
/* Use an existing CUDA stream (cudaStream_t passed as void*). */
pcg_status pcg_create_on_stream(int device, void* stream, pcg_ctx** out);
/* Drops the caller's reference.  Every object made on the context (me,
 * cells, mech, motility, batch, server, snapshot) holds one too, so the
 * context, its streams and its device status word are freed when the last
 * of them is destroyed: objects may be destroyed in any order.  The context
 * must not be used through this handle afterwards. */
pcg_status pcg_destroy(pcg_ctx* ctx);
/* MetalContext::waitForCompletion (metal_context.mm:448-461); also reports
 * PCG_ERR_DEVICE when a kernel stopped early since the last sync. */
pcg_status pcg_sync(pcg_ctx* ctx);
void* pcg_stream(pcg_ctx* ctx);
/* Orders the context's stream after every host copy issued so far by the
 * whole-batch transfers (which run on copy streams of their own, beside the
 * kernels), without waiting on the host; pcg_sync waits for them as well. */
pcg_status pcg_join(pcg_ctx* ctx);
const char* pcg_last_error_string(const pcg_ctx* ctx);
/* Number of kernel launches this context has issued (graph launches count
 * their kernel nodes). */
uint64_t pcg_kernel_launches(const pcg_ctx* ctx);
/* Page-locked host memory for the asynchronous whole-batch transfers. */
pcg_status pcg_host_alloc(size_t bytes, void** out);
pcg_status pcg_host_free(void* p);

/* ------------------------------------------------------------------------
 * Microenvironment — replaces Microenvironment (src/microenvironment.h:17-83).
 * grid->n_substrates substrates; grid->nz == 1 is the 2-D case (x and y
 * sweeps), nz > 1 adds a z sweep (decay split lambda*dt/3 per sweep) and the
 * Dirichlet reset covers all six faces.
 * ---------------------------------------------------------------------- */
pcg_status pcg_me_create(pcg_ctx* ctx, const pcg_grid_params* grid,
                         const pcg_substrate_params* substrates, pcg_me** out);
pcg_status pcg_me_destroy(pcg_me* me);
/* Microenvironment::initialize density fill (microenvironment.mm:54-60). */
pcg_status pcg_me_fill(pcg_me* me, const float* value_per_substrate);
/* Bulk setDensity / densityBuffer() read-back (microenvironment.mm:154-162);
 * n_floats must equal nx*ny*nz*S. */
pcg_status pcg_me_upload(pcg_me* me, const float* host, size_t n_floats);
pcg_status pcg_me_download(pcg_me* me, float* host, size_t n_floats);
/* Microenvironment::simulateDiffusionDecay (microenvironment.mm:106-115):
 * the x, y (, z) sweeps only, n_steps times. */
pcg_status pcg_me_diffuse(pcg_me* me, int n_steps);
/* Microenvironment::applyDirichletBC (microenvironment.mm:127-152). */
pcg_status pcg_me_apply_dirichlet(pcg_me* me);
/* processSecretion (src/cell_phenotype.cpp:526-564) for every active cell
 * of 'cells', applied per voxel in ascending cell index. */
pcg_status pcg_me_secrete(pcg_me* me, pcg_cells* cells, double dt);
/* One main-loop diffusion sub-step n_steps times (src/main.mm:341-366):
 * sweeps -> Dirichlet reset (fused into the last sweep) -> secretion (when
 * cells is not NULL), dt = grid->dt. */
pcg_status pcg_me_step(pcg_me* me, pcg_cells* cells, int n_steps);
/* Microenvironment::computeGradients + read-back (microenvironment.mm:197-257):
 * three arrays of nx*ny*nz*S floats (any may be NULL). */
pcg_status pcg_me_gradients(pcg_me* me, float* gx, float* gy, float* gz, size_t n_floats);
/* Device pointer of the density block.  On the device, rows of x are
 * row_pitch floats apart (nx rounded up to 4, so rows start on 16 bytes)
 * and substrates substrate_pitch floats apart. */
pcg_status pcg_me_device_density(pcg_me* me, float** dptr, size_t* row_pitch, size_t* substrate_pitch);

/* ------------------------------------------------------------------------
 * Cells — the GPU-shared block of CellData (src/cell_data.h:19-244).
 * ---------------------------------------------------------------------- */
pcg_status pcg_cells_create(pcg_ctx* ctx, uint32_t max_cells, uint32_t n_substrates, pcg_cells** out);
pcg_status pcg_cells_destroy(pcg_cells* cells);
/* Upload n_cells cells from a host SoA whose field stride is soa_max_cells. */
pcg_status pcg_cells_upload(pcg_cells* cells, const float* soa, uint32_t n_cells, uint32_t soa_max_cells);
pcg_status pcg_cells_download(pcg_cells* cells, float* soa, uint32_t soa_max_cells);
/* Partial transfers of fields [first, first + count). */
pcg_status pcg_cells_upload_fields(pcg_cells* cells, uint32_t first, uint32_t count,
                                   const float* soa, uint32_t soa_max_cells);
pcg_status pcg_cells_download_fields(pcg_cells* cells, uint32_t first, uint32_t count,
                                     float* soa, uint32_t soa_max_cells);
/* Per-cell per-substrate rates [cell * S + s] (n_cells * S each; NULL =
 * zeros) and the active mask (NULL = all cells; the reference skips cells
 * whose current_death_model != 0, src/main.mm:360). */
pcg_status pcg_cells_set_secretion(pcg_cells* cells, const double* secretion, const double* uptake,
                                   const double* saturation, const double* net_export,
                                   const uint8_t* active);
/* Read-back of the rates and active flags pcg_cells_set_secretion set (and
 * removals and appends moved): n_cells * S doubles each, n_cells flags (any
 * may be NULL). */
pcg_status pcg_cells_download_secretion(pcg_cells* cells, double* secretion, double* uptake, double* saturation,
                                        double* net_export, uint8_t* active);
pcg_status pcg_cells_count(pcg_cells* cells, uint32_t* n_cells);
/* Voxel index refresh.  The reference recomputes voxel_index only at
 * phenotype steps, from x and y (cell_phenotype.cpp:781-789).  With on != 0
 * every pcg_mech_integrate / pcg_mech_update on 'cells' recomputes each
 * cell's voxel_index from its new position on me's grid
 * (Microenvironment::voxelIndex, microenvironment.mm:176-184, 3-D aware),
 * and the next secretion rebuilds its order.  Off (the default) keeps the
 * indices the host set.  The batch form is PCG_INST_REFRESH_VOXELS. */
pcg_status pcg_cells_set_voxel_refresh(pcg_cells* cells, const pcg_me* me, int on);
/* Dead-cell compaction on the device, without a re-upload: CellData::
 * removeCell (src/cell_data.cpp:408-498, the last cell moved into the
 * freed place) for each of 'indices' in descending order, indices at or
 * past the current count skipped -- phase 3 of updatePhenotypes
 * (src/cell_phenotype.cpp:838-844).  Every moved cell takes its 28 SoA
 * fields, its per-substrate rates and its active flag along; the count
 * drops by the number removed.  One launch (pcg_removal_plan's moves). */
pcg_status pcg_cells_remove(pcg_cells* cells, const uint32_t* indices, uint32_t count);
/* The same removal as a list of moves, on the host only (no device work),
 * for the CPU-only per-cell arrays a host keeps: dest[k] receives the cell
 * that started at src[k], every other place below *n_final keeps its cell.
 * dest and src hold at least 'count' entries. */
pcg_status pcg_removal_plan(uint32_t n_cells, const uint32_t* indices, uint32_t count, uint32_t* dest,
                            uint32_t* src, uint32_t* n_moves, uint32_t* n_final);
/* Appends 'count' cells after the current ones, as CellData::addCell
 * (src/cell_data.cpp:398-406) places new and daughter cells: their 28
 * fields from a host SoA of field stride soa_max_cells, their per-substrate
 * rates [cell * S + s] (NULL = zeros) and active flags (NULL = active). */
pcg_status pcg_cells_append(pcg_cells* cells, const float* soa, uint32_t count, uint32_t soa_max_cells,
                            const double* secretion, const double* uptake, const double* saturation,
                            const double* net_export, const uint8_t* active);
pcg_status pcg_cells_device_soa(pcg_cells* cells, float** dptr, uint32_t* max_cells);
/* FP64 master positions.  The reference keeps positions as FP32 SoA fields
 * (integrate.metal:58-69 updates them in place); here the AB2 update runs on
 * an FP64 master copy per cell and stores its rounding into those fields.
 * The update starts from the master while the master rounds to the field's
 * FP32 value; a position the host writes through the SoA (an upload of a
 * different value, an append) replaces it.  Downloads cells [0, n_cells)
 * (n_cells = the current count) as three arrays of n_cells doubles (x, y, z),
 * each the value the next update starts from. */
pcg_status pcg_cells_download_positions64(pcg_cells* cells, double* xyz, uint32_t n_cells);

/* ------------------------------------------------------------------------
 * Mechanics — replaces CellMechanics (src/cell_mechanics.h:15-87).
 * Binning is a counting sort over the mechanics voxels, stable in cell
 * index within a voxel; the cell-start table replaces the 64-slot hash: voxelCellCount(v) =
 * start[v+1] - start[v], voxelCells(v) = sorted + start[v].
 * ---------------------------------------------------------------------- */
/* CellMechanics::initialize (cell_mechanics.mm:23-82): the mechanics
 * grid of params->mech_grid_* voxels of params->mechanics_voxel_size with
 * origin (x_min, y_min, z_min). */
pcg_status pcg_mech_create(pcg_ctx* ctx, const pcg_mechanics_params* params,
                           float x_min, float y_min, float z_min, uint32_t max_cells, pcg_mech** out);
pcg_status pcg_mech_destroy(pcg_mech* mech);
/* CellMechanics::computeForces (cell_mechanics.mm:99-111): bin, sort,
 * cell-start table, forces -> velocity and simple pressure. */
pcg_status pcg_mech_forces(pcg_mech* mech, pcg_cells* cells);
/* CellMechanics::integratePositions (cell_mechanics.mm:113-120). */
pcg_status pcg_mech_integrate(pcg_mech* mech, pcg_cells* cells, float dt);
/* CellMechanics::update (cell_mechanics.mm:84-97): forces + integrate. */
pcg_status pcg_mech_update(pcg_mech* mech, pcg_cells* cells, float dt);
/* CellMechanics::syncHashPointers (cell_mechanics.mm:122-133): copy the
 * cell-start table (V + 1 entries) and the sorted cell indices (n_cells)
 * to the host; either pointer may be NULL. */
pcg_status pcg_mech_bins(pcg_mech* mech, uint32_t* start, uint32_t* sorted_cells);
uint32_t pcg_mech_total_voxels(const pcg_mech* mech);
/* Diagnostics: when on, the force pass also records per cell the number of
 * neighbours within the cut-off and a hash of their indices (the sum of
 * pcg_neighbor_hash(j) mod 2^32), read back with pcg_mech_neighbor_stats. */
pcg_status pcg_mech_set_diagnostics(pcg_mech* mech, int on);
pcg_status pcg_mech_neighbor_stats(pcg_mech* mech, uint32_t* count, uint32_t* hash);
uint32_t pcg_neighbor_hash(uint32_t cell);

/* ------------------------------------------------------------------------
 * Motility — updateMotility (src/motility.cpp:179-293) on the device: the
 * persistent random walk with chemotaxis bias that main.mm:379-387 runs
 * between CellMechanics::computeForces and integratePositions.  State is
 * MotilityData (src/motility.h:10-50), resident on the device.
 *
 * Random draws: the reference uses an unseeded std::mt19937; here draw k of
 * cell i at step `step` is a counter-based uniform of (seed, i, step, k)
 * (k = 0 resample test, 1 theta, 2 phi), so a run is reproducible and the
 * CPU oracle computes the same draws.
 * Gradient read: layout PCG_MOT_REFERENCE reads the density as
 * motility.cpp:68-74 does (linear index voxel * n_substrates + s into the
 * substrate-major buffer); PCG_MOT_SUBSTRATE_MAJOR reads substrate s of the
 * voxel.  They agree for one substrate.
 * ---------------------------------------------------------------------- */
enum { PCG_MOT_REFERENCE = 0, PCG_MOT_SUBSTRATE_MAJOR = 1 };

/* MotilityData::allocate / allocateSubstrate (motility.cpp:90-116);
 * n_substrates = 0: the single-substrate chemotaxis rule only. */
pcg_status pcg_motility_create(pcg_ctx* ctx, uint32_t max_cells, uint32_t n_substrates, pcg_motility** out);
pcg_status pcg_motility_destroy(pcg_motility* mot);
/* Host -> device state of cells [0, n_cells): persistence_time, elapsed,
 * bias, vec (three arrays of n_cells: x, y, z), is_motile, restrict_to_2D,
 * chemotaxis_index, chemotaxis_direction, sensitivity (n_cells *
 * n_substrates, cell-major; may be NULL when created with 0 substrates). */
pcg_status pcg_motility_upload(pcg_motility* mot, uint32_t n_cells, const double* persistence_time,
                               const double* elapsed, const double* bias, const double* vec,
                               const uint32_t* is_motile, const uint32_t* restrict_2d,
                               const int32_t* chemotaxis_index, const int32_t* chemotaxis_direction,
                               const double* sensitivity);
/* Device -> host of what updateMotility changes: elapsed and vec. */
pcg_status pcg_motility_download(pcg_motility* mot, double* elapsed, double* vec);
/* updateMotility(cells, mot, density, grid, dt): adds each living motile
 * cell's motility vector to its velocity (fields 3-5, written by the force
 * pass); me supplies the density and grid for the chemotaxis gradient. */
pcg_status pcg_motility_update(pcg_motility* mot, pcg_cells* cells, const pcg_me* me, double dt, uint64_t seed,
                               uint64_t step, int layout);

/* ------------------------------------------------------------------------
 * Snapshots — writeMatlabSnapshots (src/output_writer.cpp:295-452) with
 * write_matlab4 (src/matlab_writer.cpp:5-49): MATLAB v4 files of one full
 * double matrix, byte-identical to the reference writer's.  Asynchronous:
 * the matrix is built on the device after the work queued so far on the
 * context (later work on the context waits only for that build), then
 * copied and written by a host callback while the simulation goes on.
 * Cell columns come from the 28-field SoA and the secretion rates; the
 * columns the reference takes from CPU-side phenotype arrays get the values
 * it writes when those arrays are absent.
 * ---------------------------------------------------------------------- */
pcg_status pcg_snapshot_create(pcg_ctx* ctx, pcg_snapshot** out);
/* Waits for every pending write; reports a file that could not be written. */
pcg_status pcg_snapshot_wait(pcg_snapshot* snap);
pcg_status pcg_snapshot_destroy(pcg_snapshot* snap);
/* "multiscale_microenvironment": (4 + S) x voxels, rows x, y, z, voxel
 * volume, densities. */
pcg_status pcg_snapshot_microenvironment(pcg_snapshot* snap, const pcg_me* me, const char* path);
/* "cells": (71 + 7 * types + 8 * S) x cells; n_cell_types 0 counts as 1. */
pcg_status pcg_snapshot_cells(pcg_snapshot* snap, const pcg_cells* cells, uint32_t n_cell_types, const char* path);
/* Both files of one output frame, named as the reference names them:
 * folder/output%08d_cells.mat and folder/output%08d_microenvironment0.mat
 * (either object may be NULL). */
pcg_status pcg_snapshot_frame(pcg_snapshot* snap, const pcg_me* me, const pcg_cells* cells, uint32_t n_cell_types,
                              const char* folder, int frame);

/* No reference counterpart.  A stable (key, value) radix sort -- sorting
 * mechanics-voxel keys with cell indices as values gives the cell order of
 * the mechanics binning -- run on caller-owned DEVICE buffers and making
 * no device allocation: all scratch lives in one fixed 2.5 MiB array
 * compiled into the library.  For callers that cannot allocate device
 * memory at the point of the call (a server that partitioned the device up
 * front and must not fail a request with out-of-memory, or host code that
 * must avoid allocation calls because they can synchronise the device).
 * - Sorts n pairs by the low key_bits (1..32) bits of the keys, equal keys
 *   keeping their input order; enqueued on ctx's stream (pcg_sync waits).
 *   ctx's device is made current for the call and the caller's restored.
 * - n <= PCG_SORT_STATIC_MAX_PAIRS, else PCG_ERR_INVALID with a message;
 *   outputs must not overlap the inputs or each other.
 * - The first call on each device does the device set-up: it looks up the
 *   scratch array's address and loads the sort's kernels (which lazy
 *   module loading would otherwise load, and possibly allocate for, at
 *   their first launch).  Make it, e.g. with n = 0, before the calls that
 *   matter.  The scratch needs no initial contents.
 * - One scratch array per device: calls on the same device must not
 *   overlap in time (issue them on one stream, or order them with events);
 *   overlapping calls race on the scratch and give wrong results. */
#define PCG_SORT_STATIC_MAX_PAIRS (1u << 18)
pcg_status pcg_sort_pairs_static(pcg_ctx* ctx, const uint32_t* keys_in, const uint32_t* vals_in,
                                 uint32_t* keys_out, uint32_t* vals_out, uint32_t n, int key_bits);

/* No reference counterpart (the reference aborts on a failed allocation,
 * metal_context.mm:52-60).  Test and diagnostics aids, process-wide:
 * the number of device allocations the library has made with cudaMalloc
 * and of pooled blocks it has handed out again; and a host-side fault
 * injector that makes the nth library device allocation from now fail as
 * out of memory (PCG_ERR_OOM from the call that needed it) without
 * touching the device (nth = 0 turns it off). */
void pcg_debug_alloc_stats(uint64_t* device_mallocs, uint64_t* pool_reuses);
void pcg_debug_fail_alloc(uint64_t nth);
/* No reference counterpart (a failed Metal command buffer is logged and
 * the loop goes on, metal_context.mm:448-461).  Test aid for the bounded
 * device waits: with on != 0, the first wait of every plane-sweep CTA
 * launched on ctx reports that its bound ran out at once.  The CTA records
 * it in the context's status word, waits (with the normal bound) for the
 * copies it issued and exits without storing its plane, so pcg_sync
 * returns PCG_ERR_DEVICE; with on = 0 the context works as before. */
pcg_status pcg_debug_give_up_waits(pcg_ctx* ctx, int on);

/* ------------------------------------------------------------------------
 * Batch — many independent simulations of uneven grid and cell counts
 * advanced together: one CUDA graph per main-loop step, each phase one
 * persistent kernel over a flattened work list of all instances.
 * ---------------------------------------------------------------------- */
enum { PCG_INST_REFRESH_VOXELS = 1 };   /* recompute voxel_index after integrate */

typedef struct {
    pcg_grid_params grid;                    /* diffusion grid; grid.dt = dt_diffusion */
    const pcg_substrate_params* substrates;  /* grid.n_substrates entries */
    const float* initial_density;            /* nx*ny*nz*S floats, or NULL */
    const float* initial_values;             /* per-substrate fill when initial_density is NULL */
    uint32_t n_cells;
    const float* cells_soa;                  /* 28-field SoA with stride cells_soa_max */
    uint32_t cells_soa_max;
    const double* secretion;                 /* [cell * S + s], NULL = zeros */
    const double* uptake;
    const double* saturation;
    const double* net_export;
    const uint8_t* active;                   /* NULL = all active */
    pcg_mechanics_params mech;               /* mechanics grid (cell_mechanics.mm:26-41) */
    float dt_mechanics;
    uint32_t flags;
} pcg_instance_desc;

typedef struct {
    int use_graphs;        /* capture each step into a CUDA graph (default 1) */
    int autotune;          /* pick sweep shapes, the force pass shape and the cell kernels'
                              block sizes by measurement on the batch's data (default 1) */
    const char* tune_cache;/* JSON cache path for autotuned choices, or NULL */
    int profile_phases;    /* record CUDA events around phases (default 0) */
    int pin_x;             /* launch shape of the x sweeps instead of the tuned one: */
    int pin_cols;          /* warps * 16 + stages (y and z sweeps: pin_cols); 0 = tuned */
    int disable_planes;    /* 1: x and y sweeps as separate tile passes even where an x-y plane
                              fits shared memory (same results; 0 = one pass per plane) */
    int pin_forces;        /* force pass shape instead of the tuned one: threads per block
                              (32..256, a multiple of 32) * 1000 + neighbour queue slots per
                              thread (0, 16, 32 or 64); 0 = tuned.  Same results for every shape */
    int pin_cell_threads;  /* threads per block (32..256, a multiple of 32) of the secretion,
                              binning and AB2 kernels instead of the tuned ones; 0 = tuned */
} pcg_batch_options;

pcg_status pcg_batch_create(pcg_ctx* ctx, const pcg_instance_desc* instances, uint32_t n_instances,
                            const pcg_batch_options* options, pcg_batch** out);
pcg_status pcg_batch_destroy(pcg_batch* batch);
/* Advance every instance by n_diffusion_steps main-loop sub-steps
 * (src/main.mm:341-391 ordering; mechanics when each instance's accumulator
 * reaches dt_mechanics).  One graph launch per sub-step, or per mechanics
 * period where the call covers a whole one; the same results either way. */
pcg_status pcg_batch_step(pcg_batch* batch, int n_diffusion_steps);
pcg_status pcg_batch_download_density(pcg_batch* batch, uint32_t instance, float* host, size_t n_floats);
pcg_status pcg_batch_download_cells(pcg_batch* batch, uint32_t instance, float* soa, uint32_t soa_max_cells);
pcg_status pcg_batch_upload_cells(pcg_batch* batch, uint32_t instance, const float* soa, uint32_t soa_max_cells);
/* pcg_cells_download_positions64 for one instance (n_cells = its count). */
pcg_status pcg_batch_download_positions64(pcg_batch* batch, uint32_t instance, double* xyz, uint32_t n_cells);
/* Whole-batch asynchronous transfers (the end-to-end path; host buffers
 * should come from pcg_host_alloc).  Cells: one SoA of all instances' cells
 * in instance order, field stride = total cells (28 * total floats).
 * Density: the device arena as is (pcg_batch_density_layout gives each
 * instance's offset and substrate pitch).  The host copies run on copy
 * streams through device staging buffers, so they overlap the kernels of
 * other steps: an upload is taken by the next step, a download is the state
 * at the call.  None waits for completion; pcg_sync does (pcg_join orders
 * the context stream after them). */
pcg_status pcg_batch_upload_all_cells(pcg_batch* batch, const float* soa, uint64_t n_floats);
pcg_status pcg_batch_download_all_cells(pcg_batch* batch, float* soa, uint64_t n_floats);
pcg_status pcg_batch_download_all_density(pcg_batch* batch, float* host, uint64_t n_floats);
/* pcg_batch_download_all_cells for the fields whose bit is set in
 * field_mask (bit f = field f), into the same places of the host SoA; the
 * other fields of the host SoA are left as they are.  A main loop whose host
 * keeps the fields only it writes (radius, volumes, phenotype, ...) reads
 * back PCG_STEP_WRITTEN_FIELDS: what the sub-steps and mechanics steps
 * change. */
#define PCG_STEP_WRITTEN_FIELDS                                                                   \
    ((1u << PCG_F_POS_X) | (1u << PCG_F_POS_Y) | (1u << PCG_F_POS_Z) | (1u << PCG_F_VEL_X) |      \
     (1u << PCG_F_VEL_Y) | (1u << PCG_F_VEL_Z) | (1u << PCG_F_PREV_VX) | (1u << PCG_F_PREV_VY) |  \
     (1u << PCG_F_PREV_VZ) | (1u << PCG_F_PRESSURE) | (1u << PCG_F_VOXEL_IDX) |                   \
     (1u << PCG_F_MECH_VOXEL))
pcg_status pcg_batch_download_cell_fields(pcg_batch* batch, float* soa, uint64_t n_floats, uint32_t field_mask);
/* pcg_batch_upload_all_cells for the fields whose bit is set in field_mask,
 * from the same places of the host SoA; the device's other fields are left
 * as they are.  A host that owns the phenotype fields and leaves the
 * kinematic state to the device uploads PCG_HOST_OWNED_FIELDS (every field
 * the steps do not write). */
#define PCG_HOST_OWNED_FIELDS (((1u << PCG_NUM_FIELDS) - 1u) & ~PCG_STEP_WRITTEN_FIELDS)
pcg_status pcg_batch_upload_cell_fields(pcg_batch* batch, const float* soa, uint64_t n_floats, uint32_t field_mask);
pcg_status pcg_batch_density_layout(pcg_batch* batch, uint32_t instance, uint64_t* offset, uint64_t* row_pitch,
                                    uint64_t* substrate_pitch, uint64_t* arena_floats);
/* Totals: voxels (sum nx*ny*nz), voxel-substrates, cells. */
pcg_status pcg_batch_totals(pcg_batch* batch, uint64_t* voxels, uint64_t* voxel_substrates, uint64_t* cells);
/* Voxel-substrates the sweep launches of one sub-step cover, summed over the
 * launches (each launch reads and writes every value it covers once, 8
 * bytes): those of the plane launches (fused x + y planes, x-z planes of z
 * lines), and of all sweeps. */
pcg_status pcg_batch_sweep_units(pcg_batch* batch, uint64_t* plane_units, uint64_t* all_units);
/* Kernel launches one main-loop sub-step issues: without / with a
 * mechanics step. */
pcg_status pcg_batch_step_launches(pcg_batch* batch, uint64_t* diffusion_step, uint64_t* mechanics_step);
/* Per-phase device milliseconds accumulated since the last reset when
 * profile_phases is on: [0] x sweep, [1] y sweep, [2] z sweep, [3] secretion,
 * [4] mechanics bin+sort, [5] forces, [6] integrate.  Returns the counts of
 * timed sweeps launches in *n_sweep_launches. */
#define PCG_N_PHASES 7
pcg_status pcg_batch_phase_times(pcg_batch* batch, float* ms, uint64_t* n_sweep_launches, int reset);
/* Switch phase profiling on or off after creation. */
pcg_status pcg_batch_set_profile(pcg_batch* batch, int on);
/* Neighbour-set diagnostics of the batch's force pass, as
 * pcg_mech_set_diagnostics gives them for one simulation (the mechanics
 * step's graph is captured again; results are unchanged). */
pcg_status pcg_batch_set_diagnostics(pcg_batch* batch, int on);
/* CellMechanics::syncHashPointers (cell_mechanics.mm:122-133) for one
 * instance of the batch, as of its last mechanics step: its cell-start
 * table (V + 1 entries for its V mechanics voxels, counted from its first
 * sorted place), its sorted cells (n_cells, instance-local indices) and,
 * with diagnostics on, each cell's neighbour count and hash (n_cells, by
 * instance-local cell index).  Any pointer may be NULL.  The batch's steps
 * do not need the sorted cells, so the first call after a mechanics step
 * that asks for them makes them (one kernel launch on the context stream)
 * from that step's binning. */
pcg_status pcg_batch_mech_bins(pcg_batch* batch, uint32_t instance, uint32_t* start, uint32_t* sorted_cells,
                               uint32_t* nbr_count, uint32_t* nbr_hash);
/* Describe the chosen launch shapes as a short string. */
const char* pcg_batch_describe(pcg_batch* batch);

/* ------------------------------------------------------------------------
 * Serving — continuous batching of parameter-sweep simulations.  Requests
 * are admitted against a device-memory budget as slots and memory free up,
 * their state stays resident on the device, and all admitted requests
 * advance together in chunks of steps.
 * ---------------------------------------------------------------------- */
typedef struct {
    uint64_t budget_bytes;     /* device bytes requests may hold (e.g. 150e9) */
    uint32_t max_active;       /* slot limit, 0 = unlimited */
    uint32_t steps_per_tick;   /* diffusion sub-steps per tick (default 100) */
} pcg_serve_options;

enum { PCG_REQ_QUEUED = 0, PCG_REQ_RUNNING = 1, PCG_REQ_DONE = 2, PCG_REQ_CANCELLED = 3 };

pcg_status pcg_serve_create(pcg_ctx* ctx, const pcg_serve_options* options, pcg_server** out);
/* One server over several contexts, normally one per GPU (a device may
 * also appear more than once).  Each request runs on one context, chosen
 * when it is admitted: the one with the most unused budget among those
 * where it fits.  budget_bytes and max_active apply to each context.
 * Every context's sub-steps of a tick are issued before any is waited for,
 * so the GPUs work at the same time.  The contexts are used from the
 * calling thread only; each is made current while its work is issued. */
pcg_status pcg_serve_create_multi(pcg_ctx* const* ctxs, uint32_t n_ctx, const pcg_serve_options* options,
                                  pcg_server** out);
pcg_status pcg_serve_destroy(pcg_server* srv);
/* Queue a request (the host data is copied); *id receives its id. */
pcg_status pcg_serve_submit(pcg_server* srv, const pcg_instance_desc* inst, uint32_t n_diffusion_steps,
                            uint64_t* id);
/* Admit what fits, advance every running request by one chunk, retire the
 * finished ones.  *n_running / *n_queued / *n_finished_now may be NULL. */
pcg_status pcg_serve_tick(pcg_server* srv, uint32_t* n_running, uint32_t* n_queued, uint32_t* n_finished_now);
pcg_status pcg_serve_state(pcg_server* srv, uint64_t id, int* state);
/* Cancels a request: a queued one leaves the queue now, a running one
 * leaves its batch (and frees its budget) at the next tick; its state
 * becomes PCG_REQ_CANCELLED and fetch / request_times refuse it.  A finished
 * request cannot be cancelled (PCG_ERR_INVALID). */
pcg_status pcg_serve_cancel(pcg_server* srv, uint64_t id);
/* Index (into the contexts the server was made with) of the context a
 * request was admitted to, -1 while it is queued. */
pcg_status pcg_serve_placement(pcg_server* srv, uint64_t id, int* ctx_index);
/* Results of a finished request; either pointer may be NULL. */
pcg_status pcg_serve_fetch(pcg_server* srv, uint64_t id, float* density, size_t n_floats,
                           float* soa, uint32_t soa_max_cells);
/* Device seconds and wall seconds a request spent, from admission and from
 * submission to completion. */
pcg_status pcg_serve_request_times(pcg_server* srv, uint64_t id, double* submit_to_done_s,
                                   double* admit_to_done_s);
/* Totals since creation: voxel-steps, cell-steps (mechanics), bytes held now. */
pcg_status pcg_serve_totals(pcg_server* srv, uint64_t* voxel_steps, uint64_t* cell_steps,
                            uint64_t* bytes_in_use);
/* Bytes the library would hold for one request (admission estimate). */
uint64_t pcg_instance_bytes(const pcg_instance_desc* inst);

#ifdef __cplusplus
}
#endif
#endif /* PCG_H */
