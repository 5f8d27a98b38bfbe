/*
 * ref_wrap.cpp — C entry points that run the reference's own code on the
 * CPU (TEST INFRASTRUCTURE: builds oracle/_ref/libpcg_ref.so, the checker
 * for the oracle; nothing in the product links it).
 *
 * Compiled together with, from the reference tree as they lie:
 *   shaders/diffusion_2d.metal, shaders/mechanics.metal, shaders/integrate.metal
 *     (through metal_shim.h; one call per Metal thread id, ascending, so the
 *     spatial-hash slot order is ascending cell index)
 *   src/cell_phenotype.cpp (processSecretion), src/cell_data.cpp,
 *   src/cell_definitions.cpp, src/motility.cpp (updateMotility),
 *   src/output_writer.cpp + src/matlab_writer.cpp (writeMatlabSnapshots)
 * The host-side steps that live in Objective-C++ files and cannot be
 * compiled here are restated below with their citations:
 *   ThomasCoeffs set-up   src/microenvironment.mm:86-92
 *   applyDirichletBC      src/microenvironment.mm:127-152
 */
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <vector>
#include <atomic>

#include "types.h"
#include "cell_data.h"
#include "cell_phenotype.h"
#include "motility.h"
#include "output_writer.h"

#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::atomic<uint32_t> atomic_uint_t;

// kernels from the reference shaders (compiled as C++ via metal_shim.h)
void diffusion_sweep_x(float*, const GridParams&, const SubstrateParams*, const ThomasCoeffs*, unsigned int);
void diffusion_sweep_y(float*, const GridParams&, const SubstrateParams*, const ThomasCoeffs*, unsigned int);
void clear_spatial_hash(atomic_uint_t*, const unsigned int&, unsigned int);
void build_spatial_hash(float*, atomic_uint_t*, unsigned int*, const MechanicsParams&, const GridParams&,
                        const unsigned int&, const unsigned int&, unsigned int);
void compute_forces(float*, atomic_uint_t*, unsigned int*, const MechanicsParams&, const unsigned int&,
                    const unsigned int&, unsigned int);
void integrate_positions(float*, const GridParams&, const float&, const unsigned int&, const unsigned int&,
                         unsigned int);

extern "C" {

int ref_sizeof_grid(void) { return (int)sizeof(GridParams); }
int ref_sizeof_substrate(void) { return (int)sizeof(SubstrateParams); }
int ref_sizeof_mech(void) { return (int)sizeof(MechanicsParams); }
int ref_max_cells_per_voxel(void) { return MAX_CELLS_PER_VOXEL; }

/* microenvironment.mm:86-92 */
void ref_thomas_coeffs(const GridParams* g, const SubstrateParams* sp, ThomasCoeffs* tc)
{
    for (uint32_t s = 0; s < g->n_substrates; s++) {
        float D = sp[s].diffusion_coefficient;
        float lambda = sp[s].decay_rate;
        float dt = g->dt;
        tc[s].coeff = D * dt / (g->dx * g->dx);
        tc[s].half_decay = 0.5f * lambda * dt;
        tc[s]._pad[0] = tc[s]._pad[1] = 0.0f;
    }
}

/* Microenvironment::simulateDiffusionDecay: x then y (microenvironment.mm:106-115). */
void ref_simulate_diffusion_decay(float* density, const GridParams* g, const SubstrateParams* sp, int threads)
{
    std::vector<ThomasCoeffs> tc(g->n_substrates ? g->n_substrates : 1);
    ref_thomas_coeffs(g, sp, tc.data());
    const long long ny = g->ny, nx = g->nx;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
    #pragma omp parallel for schedule(static) if (threads != 1)
#endif
    for (long long t = 0; t < ny; t++) diffusion_sweep_x(density, *g, sp, tc.data(), (unsigned)t);
#ifdef _OPENMP
    #pragma omp parallel for schedule(static) if (threads != 1)
#endif
    for (long long t = 0; t < nx; t++) diffusion_sweep_y(density, *g, sp, tc.data(), (unsigned)t);
}

void ref_sweep_x(float* density, const GridParams* g, const SubstrateParams* sp)
{
    std::vector<ThomasCoeffs> tc(g->n_substrates ? g->n_substrates : 1);
    ref_thomas_coeffs(g, sp, tc.data());
    for (uint32_t t = 0; t < g->ny; t++) diffusion_sweep_x(density, *g, sp, tc.data(), t);
}

void ref_sweep_y(float* density, const GridParams* g, const SubstrateParams* sp)
{
    std::vector<ThomasCoeffs> tc(g->n_substrates ? g->n_substrates : 1);
    ref_thomas_coeffs(g, sp, tc.data());
    for (uint32_t t = 0; t < g->nx; t++) diffusion_sweep_y(density, *g, sp, tc.data(), t);
}

/* microenvironment.mm:127-152 */
void ref_apply_dirichlet(float* density, const GridParams* g, const SubstrateParams* sp)
{
    const uint32_t nx = g->nx, ny = g->ny, total = nx * ny * g->nz;
    for (uint32_t s = 0; s < g->n_substrates; s++) {
        if (!sp[s].dirichlet_enabled) continue;
        float target = sp[s].target_value;
        uint32_t base = s * total;
        for (uint32_t i = 0; i < nx; i++) { density[base + i] = target; density[base + (ny - 1) * nx + i] = target; }
        for (uint32_t j = 0; j < ny; j++) { density[base + j * nx] = target; density[base + j * nx + nx - 1] = target; }
    }
}

/* processSecretion (cell_phenotype.cpp:526-564) for every cell in ascending
 * index.  Arrays are the CellData fields it reads. */
void ref_process_secretion(float* density, const GridParams* g, uint32_t n_cells,
                           const uint32_t* voxel, const float* volume,
                           const double* sec, const double* upt, const double* sat, const double* ne,
                           double dt)
{
    CellData cells(n_cells ? n_cells : 1);
    std::vector<float> block(cells.gpuBufferSize() / sizeof(float), 0.0f);
    cells.setGPUBufferBase(block.data());
    cells.allocateSubstrateBuffers(g->n_substrates);
    cells.num_cells = n_cells;
    const size_t nS = (size_t)n_cells * g->n_substrates;
    for (uint32_t i = 0; i < n_cells; i++) { cells.voxel_index[i] = voxel[i]; cells.total_volume[i] = volume[i]; }
    std::memcpy(cells.secretion_rate, sec, nS * sizeof(double));
    std::memcpy(cells.uptake_rate, upt, nS * sizeof(double));
    std::memcpy(cells.saturation_density, sat, nS * sizeof(double));
    std::memcpy(cells.net_export_rate, ne, nS * sizeof(double));
    for (uint32_t i = 0; i < n_cells; i++) processSecretion(cells, density, *g, i, dt);
}

/* CellMechanics::computeForces pipeline (metal_context.mm:390-443):
 * clear -> build -> forces, thread ids ascending.  hash_counts has
 * n_voxels entries, hash_cells n_voxels * 64. */
void ref_compute_forces(float* soa, uint32_t max_cells, uint32_t n_cells, const MechanicsParams* m,
                        const GridParams* mech_grid, uint32_t* hash_counts, uint32_t* hash_cells, int threads)
{
    const uint32_t V = m->mech_grid_nx * m->mech_grid_ny * m->mech_grid_nz;
    atomic_uint_t* counts = reinterpret_cast<atomic_uint_t*>(hash_counts);
    for (uint32_t t = 0; t < V; t++) clear_spatial_hash(counts, V, t);
    for (uint32_t t = 0; t < n_cells; t++)
        build_spatial_hash(soa, counts, hash_cells, *m, *mech_grid, n_cells, max_cells, t);
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
    #pragma omp parallel for schedule(dynamic, 256) if (threads != 1)
#endif
    for (long long t = 0; t < (long long)n_cells; t++)
        compute_forces(soa, counts, hash_cells, *m, n_cells, max_cells, (unsigned)t);
}

void ref_integrate(float* soa, uint32_t max_cells, uint32_t n_cells, const GridParams* mech_grid, float dt)
{
    for (uint32_t t = 0; t < n_cells; t++) integrate_positions(soa, *mech_grid, dt, n_cells, max_cells, t);
}

/* updateMotility (motility.cpp:179-293) on a 28-field SoA block and the
 * MotilityData arrays (vec: three arrays of n_cells).  Its random draws come
 * from the reference's own unseeded generator, so only results that do not
 * depend on them are comparable (bias 1 with persistence below dt). */
void ref_update_motility(float* soa, uint32_t max_cells, uint32_t n_cells, const float* density, const GridParams* g,
                         double* persistence, double* elapsed, const double* bias, double* vec,
                         const uint32_t* is_motile, const uint32_t* restrict_2d, const int32_t* chem_index,
                         const int32_t* chem_dir, const double* sens, uint32_t n_sens, double dt)
{
    CellData cells(max_cells ? max_cells : 1);
    std::vector<float> block(cells.gpuBufferSize() / sizeof(float), 0.0f);
    std::memcpy(block.data(), soa, (size_t)NUM_CELL_FIELDS * max_cells * sizeof(float));
    cells.setGPUBufferBase(block.data());
    cells.num_cells = n_cells;
    MotilityData mot;
    mot.allocate(max_cells ? max_cells : 1);
    if (sens && n_sens) mot.allocateSubstrate(n_sens);
    for (uint32_t i = 0; i < n_cells; i++) {
        mot.persistence_time[i] = persistence[i];
        mot.motility_elapsed[i] = elapsed[i];
        mot.motility_bias[i] = bias[i];
        mot.motility_vec_x[i] = vec[i];
        mot.motility_vec_y[i] = vec[n_cells + i];
        mot.motility_vec_z[i] = vec[2 * (size_t)n_cells + i];
        mot.is_motile[i] = is_motile[i];
        mot.restrict_to_2D[i] = restrict_2d[i];
        mot.chemotaxis_index[i] = chem_index[i];
        mot.chemotaxis_direction[i] = chem_dir[i];
        for (uint32_t s = 0; sens && s < n_sens; s++)
            mot.chemotactic_sensitivity[(size_t)i * n_sens + s] = sens[(size_t)i * n_sens + s];
    }
    updateMotility(cells, mot, density, *g, dt);
    std::memcpy(soa, block.data(), (size_t)NUM_CELL_FIELDS * max_cells * sizeof(float));
    for (uint32_t i = 0; i < n_cells; i++) {
        persistence[i] = mot.persistence_time[i];
        elapsed[i] = mot.motility_elapsed[i];
        vec[i] = mot.motility_vec_x[i];
        vec[n_cells + i] = mot.motility_vec_y[i];
        vec[2 * (size_t)n_cells + i] = mot.motility_vec_z[i];
    }
    mot.free_all();
}

/* writeMatlabSnapshots (output_writer.cpp:295-452) of a CellData holding
 * the 28-field SoA block and the secretion rates only (its CPU-side
 * phenotype arrays absent, so the writer uses its defaults for them), and a
 * substrate-major density; files output%08d_cells.mat and
 * output%08d_microenvironment0.mat in 'folder'. */
void ref_write_matlab(const float* soa, uint32_t max_cells, uint32_t n_cells, uint32_t n_cell_types,
                      const double* sec, const double* upt, const double* sat, const double* ne,
                      const float* density, const GridParams* g, int frame, const char* folder)
{
    CellData cells(max_cells ? max_cells : 1);
    std::vector<float> block(cells.gpuBufferSize() / sizeof(float), 0.0f);
    std::memcpy(block.data(), soa, (size_t)NUM_CELL_FIELDS * max_cells * sizeof(float));
    cells.setGPUBufferBase(block.data());
    cells.num_cells = n_cells;
    cells.num_cell_types = n_cell_types;
    cells.allocateSubstrateBuffers(g->n_substrates);
    const size_t nS = (size_t)n_cells * g->n_substrates;
    std::memcpy(cells.secretion_rate, sec, nS * sizeof(double));
    std::memcpy(cells.uptake_rate, upt, nS * sizeof(double));
    std::memcpy(cells.saturation_density, sat, nS * sizeof(double));
    std::memcpy(cells.net_export_rate, ne, nS * sizeof(double));
    writeMatlabSnapshots(cells, density, *g, frame, folder);
}

/* Phase 3 of updatePhenotypes (cell_phenotype.cpp:838-844, restated: the
 * dead-cell indices sorted descending, those at or past num_cells skipped)
 * over the reference's own CellData::removeCell (cell_data.cpp:408-498), on
 * a CellData holding the 28-field SoA block and the four per-substrate rate
 * arrays (its CPU-only phenotype arrays absent, which removeCell skips).
 * soa and the rate arrays (max_cells * S each) are updated in place;
 * returns the new count. */
uint32_t ref_remove_cells(float* soa, uint32_t max_cells, uint32_t n_cells, uint32_t n_substrates,
                          double* sec, double* upt, double* sat, double* ne,
                          const uint32_t* indices, uint32_t count)
{
    CellData cells(max_cells ? max_cells : 1);
    std::vector<float> block(cells.gpuBufferSize() / sizeof(float), 0.0f);
    std::memcpy(block.data(), soa, (size_t)NUM_CELL_FIELDS * max_cells * sizeof(float));
    cells.setGPUBufferBase(block.data());
    cells.num_cells = n_cells;
    const size_t nS = (size_t)max_cells * n_substrates;
    if (n_substrates) {
        cells.allocateSubstrateBuffers(n_substrates);
        std::memcpy(cells.secretion_rate, sec, nS * sizeof(double));
        std::memcpy(cells.uptake_rate, upt, nS * sizeof(double));
        std::memcpy(cells.saturation_density, sat, nS * sizeof(double));
        std::memcpy(cells.net_export_rate, ne, nS * sizeof(double));
    }
    std::vector<uint32_t> to_remove(indices, indices + count);
    std::sort(to_remove.begin(), to_remove.end(), std::greater<uint32_t>());
    for (uint32_t idx : to_remove)
        if (idx < cells.num_cells) cells.removeCell(idx);
    std::memcpy(soa, block.data(), (size_t)NUM_CELL_FIELDS * max_cells * sizeof(float));
    if (n_substrates) {
        std::memcpy(sec, cells.secretion_rate, nS * sizeof(double));
        std::memcpy(upt, cells.uptake_rate, nS * sizeof(double));
        std::memcpy(sat, cells.saturation_density, nS * sizeof(double));
        std::memcpy(ne, cells.net_export_rate, nS * sizeof(double));
    }
    return cells.num_cells;
}

}  // extern "C"
