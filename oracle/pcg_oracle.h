/*
 * pcg_oracle.h — CPU oracle for the per-step hot path (TEST INFRASTRUCTURE).
 *
 * This library is the checker, never the product: only tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline leg of bench.py load it.
 * The product path (libpcg.so) never links or calls anything declared here.
 *
 * It restates, in plain C, the arithmetic of the reference's hot path:
 *   - LOD Thomas sweeps          shaders/diffusion_2d.metal:28-157 (x), :165-292 (y)
 *   - Dirichlet edge reset       src/microenvironment.mm:127-152 (applyDirichletBC)
 *   - secretion / uptake         src/cell_phenotype.cpp:526-564 (processSecretion)
 *   - spatial-hash binning       shaders/mechanics.metal:41-85 (build_spatial_hash)
 *   - neighbour forces           shaders/mechanics.metal:91-216 (compute_forces)
 *   - AB2 position update        shaders/integrate.metal:31-80 (integrate_positions)
 *   - mechanics grid set-up      src/cell_mechanics.mm:23-82 (CellMechanics::initialize)
 *   - sub-step ordering          src/main.mm:341-391
 *
 * Precision modes for the diffusion sweeps:
 *   OR_FP64      — every line solved in double from the stored FP32 values and
 *                  rounded to FP32 once per sweep (where the reference stores);
 *                  this is the parity oracle.
 *   OR_FP32_REF  — the reference's own FP32 operation sequence (divisions,
 *                  in-place d' storage), IEEE round-to-nearest, no contraction;
 *                  used to show the restatement is faithful op-by-op.
 *
 * Determinism rules the reference leaves open (its GPU hash and its secretion
 * loop are racy):
 *   - secretion is applied cell by cell in ascending cell index;
 *   - cells inside one mechanics voxel are visited in ascending cell index,
 *     neighbour voxels in dk -> dj -> di order;
 *   - there is no 64-cells-per-voxel cap (tests check occupancy <= 64 where
 *     the reference semantics must coincide).
 *
 * 3-D rule (the reference sweeps x and y of the z = 0 slab only): sweeps run
 * x -> y -> z with the same per-line rule, the decay is split lambda*dt/3 per
 * sweep (lambda*dt/2 in 2-D, the reference's half_decay), and the Dirichlet
 * reset covers all six faces.  Parity for 3-D is therefore pinned by the 2-D
 * reference runs plus the pure-decay known answer rho/(1+lambda*dt/3)^3.
 */
#ifndef PCG_ORACLE_H
#define PCG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same memory layout as the reference's GridParams / SubstrateParams /
 * MechanicsParams (shaders/types.h:23-61). */
typedef struct {
    uint32_t nx, ny, nz, n_substrates;
    float dx, dy, dz, dt;
    float x_min, y_min, z_min, _pad0;
} or_grid;

/* dirichlet_consistent (the library's option, not the reference's): on
 * Dirichlet lines the end interior nodes take the interior diagonal
 * 1 + 2c + hd instead of 1 + c + hd (OR_FP64 only). */
typedef struct {
    float diffusion_coefficient, decay_rate, supply_rate, target_value;
    uint32_t dirichlet_enabled;
    uint32_t dirichlet_consistent;
    float _pad[2];
} or_substrate;

typedef struct {
    float dt, cell_cell_repulsion, cell_cell_adhesion, max_interaction_distance;
    float mechanics_voxel_size;
    uint32_t mech_grid_nx, mech_grid_ny, mech_grid_nz;
} or_mech;

enum { OR_FP64 = 0, OR_FP32_REF = 1 };

/* Cell SoA field ids (shaders/types.h:74-102). */
enum {
    OR_F_POS_X = 0, OR_F_POS_Y = 1, OR_F_POS_Z = 2,
    OR_F_VEL_X = 3, OR_F_VEL_Y = 4, OR_F_VEL_Z = 5,
    OR_F_PREV_VX = 6, OR_F_PREV_VY = 7, OR_F_PREV_VZ = 8,
    OR_F_RADIUS = 9, OR_F_TOTAL_VOL = 11,
    OR_F_REPULSION = 13, OR_F_ADHESION = 14, OR_F_REL_MAX_ADH = 15,
    OR_F_PRESSURE = 22, OR_F_VOXEL_IDX = 26, OR_F_MECH_VOXEL = 27,
    OR_NUM_FIELDS = 28
};

/* ---- diffusion ------------------------------------------------------- */

/* One diffusion-decay step on density[s][k][j][i] (FP32 storage): sweeps
 * x, y (and z when nz > 1).  The decay split is lambda*dt/d with d the number
 * of sweeps.  'mode' is OR_FP64 or OR_FP32_REF.  Does not apply the
 * Dirichlet reset (the reference calls it separately). */
void or_diffusion_sweeps(float* density, const or_grid* g, const or_substrate* subs, int mode);

/* Only the x sweep / only the y sweep / only the z sweep. */
void or_sweep_axis(float* density, const or_grid* g, const or_substrate* subs, int axis, int mode);

/* applyDirichletBC: 2-D (nz == 1) resets the four edges of the slab; 3-D
 * resets all six faces. */
void or_apply_dirichlet(float* density, const or_grid* g, const or_substrate* subs);

/* Gradients (Microenvironment::computeGradients, microenvironment.mm:197-257),
 * computed in double from FP32 density, stored FP32. */
void or_gradients(const float* density, const or_grid* g, float* gx, float* gy, float* gz);

/* ---- secretion ------------------------------------------------------- */

/* processSecretion for every cell in ascending index.  voxel[i] is the
 * cell's diffusion voxel, volume[i] its total volume (FP32), the four rate
 * arrays are [cell * S + s] (FP64), active[i] != 0 selects the cell (NULL =
 * all).  Cells whose voxel is out of range are skipped. */
void or_secretion(float* density, const or_grid* g, uint32_t n_cells,
                  const uint32_t* voxel, const float* volume,
                  const double* secretion, const double* uptake,
                  const double* saturation, const double* net_export,
                  const uint8_t* active, double dt);

/* ---- mechanics ------------------------------------------------------- */

/* CellMechanics::initialize mech-grid rule (30 um voxel, truncation, nz = 1
 * in 2-D). */
void or_mech_params(float x_min, float x_max, float y_min, float y_max,
                    float z_min, float z_max, int use_2d, float dt_mech, or_mech* out);

/* Bin every cell (mechanics.metal:54-76): key[i] = linear mech voxel.  Writes
 * the key into field OR_F_MECH_VOXEL as uint bits, like the reference. */
void or_mech_bin(float* soa, uint32_t max_cells, uint32_t n_cells, const or_mech* m,
                 float x_min, float y_min, float z_min, uint32_t* key);

/* Stable sort by key: order[p] = cell at sorted position p, start[v] =
 * first sorted position of voxel v (V + 1 entries). */
void or_mech_sort(const uint32_t* key, uint32_t n_cells, uint32_t n_voxels,
                  uint32_t* order, uint32_t* start);

/* Forces (mechanics.metal:91-216) in double from FP32 inputs; writes
 * velocity (= force) and simple pressure as FP32.  Neighbour decisions
 * (cut-off, self, 1e-12 floor) use the reference's FP32 dist_sq so that
 * neighbour sets are exact.  Optional outputs (may be NULL): nbr_count[i] =
 * neighbours within the cut-off, nbr_hash[i] = sum over neighbours j of
 * or_nbr_hash(j) (mod 2^32), force_scale[i] = sum of the magnitudes of the
 * repulsion and adhesion terms
 * (used for relative tolerances). */
void or_mech_forces(float* soa, uint32_t max_cells, uint32_t n_cells, const or_mech* m,
                    const uint32_t* key, const uint32_t* order, const uint32_t* start,
                    uint32_t* nbr_count, uint32_t* nbr_hash, double* force_scale);

uint32_t or_nbr_hash(uint32_t j);

/* AB2 update (integrate.metal:31-80) in double, stored FP32; clamp box is
 * the mechanics grid [min, min + n * voxel] (cell_mechanics.mm:57-70). */
void or_mech_integrate(float* soa, uint32_t max_cells, uint32_t n_cells, const or_mech* m,
                       float x_min, float y_min, float z_min, float dt);

/* The same update on FP64 master positions pos64 (three arrays of
 * max_cells: x, y, z), the FP32 SoA positions being their rounding.  A
 * master is the starting point when it rounds to the SoA's FP32 value;
 * otherwise (the FP32 position was written by someone else, or the master
 * was never set) the FP32 value is.  The result is stored in both.
 * pos64 = NULL is or_mech_integrate. */
void or_mech_integrate_master(float* soa, uint32_t max_cells, uint32_t n_cells, const or_mech* m,
                              float x_min, float y_min, float z_min, float dt, double* pos64);

/* Voxel refresh from positions (3-D aware form of cell_phenotype.cpp:781-789):
 * voxel_index = Microenvironment::voxelIndex(x, y, z) (microenvironment.mm:176-184). */
void or_voxel_refresh(float* soa, uint32_t max_cells, uint32_t n_cells, const or_grid* g);

/* Dead-cell compaction: phase 3 of updatePhenotypes (cell_phenotype.cpp:
 * 837-844) -- indices sorted descending, those at or past the current count
 * skipped -- over CellData::removeCell (cell_data.cpp:408-498), which moves
 * the last cell into the freed place.  Moves the 28 SoA fields (as bits),
 * the four per-substrate rate arrays [cell * S + s] and active[] (any of
 * those may be NULL); returns the new count. */
uint32_t or_cells_remove(float* soa, uint32_t max_cells, uint32_t n_cells, uint32_t S, double* sec, double* upt,
                         double* sat, double* ne, uint8_t* active, const uint32_t* indices, uint32_t count);

/* ---- whole step (main.mm:341-391 ordering, hot path only) ------------ */

typedef struct {
    or_grid grid;                 /* diffusion grid; grid.dt = dt_diffusion */
    const or_substrate* subs;     /* n_substrates entries */
    or_mech mech;                 /* mechanics grid */
    float dt_mechanics;
    int refresh_voxels;           /* recompute voxel_index after integrate */
    double* pos64;                /* FP64 master positions (or_mech_integrate_master), or NULL */
} or_sim;

/* ---------------------------------------------------------------- motility
 *
 * updateMotility (src/motility.cpp:179-293): persistent random walk with a
 * chemotaxis bias, added to the velocity the force pass wrote.  The
 * reference draws from a std::mt19937 seeded by std::random_device, which
 * cannot be reproduced; here every draw is or_uniform(seed, cell, step, k)
 * with k = 0 (resample test), 1 (theta), 2 (phi), a counter-based
 * generator the device uses too.  Parity with the reference itself is
 * pinned where its result does not depend on the draws: bias 1 with
 * persistence below dt makes every motile cell's vector the normalised
 * gradient times its speed.
 *
 * Gradient read (motility.cpp:46-87): the reference indexes the density as
 * density[voxel * n_substrates + s] although the buffer is substrate-major;
 * layout OR_MOT_REF reproduces that, OR_MOT_SUBSTRATE_MAJOR reads
 * density[s * n_voxels + voxel].  The two agree for one substrate. */
enum { OR_MOT_REF = 0, OR_MOT_SUBSTRATE_MAJOR = 1 };

/* Per-cell motility state (src/motility.h:10-50), arrays of n_cells; vec is
 * three arrays of n_cells (x, y, z).  sensitivity: n_cells * n_sens doubles
 * or NULL for the single-substrate rule (chemotaxis_index / direction). */
typedef struct {
    double* persistence_time;
    double* elapsed;
    const double* bias;
    double* vec;
    const uint32_t* is_motile;
    const uint32_t* restrict_2d;
    const int32_t* chemotaxis_index;
    const int32_t* chemotaxis_direction;
    const double* sensitivity;
    uint32_t n_sens;
} or_motility;

/* Uniform double in [0, 1) of draw k for (seed, cell, step): three rounds
 * of the SplitMix64 finaliser (Steele, Lea and Flood, 2014), 53 bits. */
double or_uniform(uint64_t seed, uint64_t cell, uint64_t step, uint32_t k);

/* soa: 28-field SoA (velocity fields 3-5 updated, speed field 16 and
 * is_alive field 25 read); density: substrate-major FP32 of grid g. */
void or_motility_update(float* soa, uint32_t max_cells, uint32_t n_cells, const float* density,
                        const or_grid* g, or_motility* mot, double dt, uint64_t seed, uint64_t step,
                        int layout);

/* Runs n_diffusion_steps of: sweeps -> Dirichlet -> secretion ->
 * [mech accumulator: bin/sort -> forces -> integrate].  mech_accum carries
 * the accumulator between calls (start at 0). */
void or_run(const or_sim* sim, float* density, float* soa, uint32_t max_cells, uint32_t n_cells,
            const double* secretion, const double* uptake, const double* saturation,
            const double* net_export, const uint8_t* active,
            int n_diffusion_steps, double* mech_accum);

/* or_run with the motility phase of main.mm:379-387: forces -> motility
 * update (dt = dt_mechanics, draw step *mot_step, then *mot_step + 1) ->
 * integrate.  mot = NULL is or_run. */
void or_run_motile(const or_sim* sim, float* density, float* soa, uint32_t max_cells, uint32_t n_cells,
                   const double* secretion, const double* uptake, const double* saturation,
                   const double* net_export, const uint8_t* active,
                   int n_diffusion_steps, double* mech_accum,
                   or_motility* mot, uint64_t seed, uint64_t* mot_step, int layout);

#ifdef __cplusplus
}
#endif
#endif
