// pcg_host.h — C++ drop-ins for the reference's Microenvironment and
// CellMechanics classes (src/microenvironment.h:17-83,
// src/cell_mechanics.h:15-87), for MotilityData / updateMotility
// (src/motility.h:20-81) and for writeMatlabSnapshots
// (src/output_writer.h:51-53), implemented over the C ABI of include/pcg.h.
//
// The public methods keep the reference's names, arguments and meaning.
// The configuration and cell store are template parameters so that the
// reference's own SimConfig (src/config_parser.h:136-177) and CellData
// (src/cell_data.h:19-244) plug in unchanged; pcg::SimConfig and
// pcg::CellStore below carry just the members these classes read.
//
// Memory model.  The reference shares one buffer between CPU and GPU
// (Apple UMA).  Here the state lives on the device and a host mirror is kept
// for the calls that hand out host pointers (densityBuffer(), the CellData
// block): a host pointer handed out marks the mirror as possibly written,
// and the next device operation uploads it first.  Callers that stay on the
// device path (step(), secreteAll()) never copy.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "pcg.h"

namespace pcg {

struct SubstrateConfig {
    std::string name;
    float diffusion_coeff = 0.0f;
    float decay_rate = 0.0f;
    float initial_value = 0.0f;
    bool dirichlet_enabled = false;
    float dirichlet_value = 0.0f;
};

struct SimConfig {
    pcg_grid_params grid{};          // grid.dx / dy / dz are read
    float x_min = 0, x_max = 0, y_min = 0, y_max = 0, z_min = 0, z_max = 0;
    bool use_2D = true;
    float dt_diffusion = 0.01f;
    float dt_mechanics = 0.1f;
    std::vector<SubstrateConfig> substrates;
};

// The GPU-shared part of CellData: 28 float/uint fields of max_cells each
// (src/cell_data.cpp:101-180) plus the per-cell per-substrate rates.
struct CellStore {
    explicit CellStore(uint32_t max_cells, uint32_t n_substrates = 0);
    uint32_t num_cells = 0;
    uint32_t max_cells = 0;
    uint32_t n_substrates = 0;
    uint32_t num_cell_types = 1;
    std::vector<float> block;        // [field * max_cells + cell]
    float* position_x = nullptr;     // == block.data(), as in CellData
    std::vector<double> secretion_rate, uptake_rate, saturation_density, net_export_rate;
    std::vector<uint32_t> current_death_model;
    float* field(int f) { return block.data() + static_cast<size_t>(f) * max_cells; }
    uint32_t addCell();
};

class Error : public std::runtime_error {
public:
    Error(int status, const std::string& what) : std::runtime_error(what), status(status) {}
    int status;
};

struct MotilityData;

// Replaces MetalContext (src/metal_context.h:14-100).  Device state made
// for host-side objects that may outlive it (MotilityData's device copy, the
// device cell stores) is released when the Context goes.
class Context {
public:
    explicit Context(int device = 0);
    ~Context();
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    pcg_ctx* get() const { return ctx_; }
    void waitForCompletion();
    void check(int status) const;
private:
    friend struct MotilityData;
    pcg_ctx* ctx_ = nullptr;
    std::vector<MotilityData*> motility_;
};

class Microenvironment {
public:
    Microenvironment() = default;
    ~Microenvironment();

    template <class Config>
    void initialize(const Config& config, Context* ctx);

    // x, y (, z) sweeps on the device (microenvironment.mm:106-115)
    void simulateDiffusionDecay();
    // microenvironment.mm:127-152
    void applyDirichletBC();
    // One main-loop diffusion sub-step on the device: sweeps, Dirichlet reset
    // and secretion of every active cell (main.mm:341-363).
    template <class Cells>
    void step(Cells& cells);
    // processSecretion for all cells at once, ascending cell index per voxel
    template <class Cells>
    void secreteAll(Cells& cells, double dt);

    float getDensity(uint32_t voxel_index, uint32_t substrate_index) const;
    void setDensity(uint32_t voxel_index, uint32_t substrate_index, float value);
    // microenvironment.mm:164-174 (single voxel, CPU formula, on the mirror)
    void applySecretion(uint32_t voxel_index, uint32_t substrate_index, float secretion_rate, float uptake_rate,
                        float saturation_density, float dt);

    uint32_t numVoxels() const { return grid_.nx * grid_.ny * grid_.nz; }
    uint32_t voxelIndex(float x, float y, float z) const;   // microenvironment.mm:176-184
    pcg_grid_params getGridParams() const { return grid_; }
    Context* context() const { return ctx_; }

    void computeGradients();
    void getGradient(uint32_t voxel_index, uint32_t substrate_index, float& gx, float& gy, float& gz) const;
    float* gradientX() { return gx_.data(); }
    float* gradientY() { return gy_.data(); }
    float* gradientZ() { return gz_.data(); }

    // Host view of the density (read back from the device); writes through
    // it reach the device before the next device operation.
    float* densityBuffer();
    const pcg_substrate_params* substrateParams() const { return subs_.data(); }
    pcg_me* handle() const { return me_; }

    // keeps the host mirror and the device consistent before a device call
    void push_host_writes();
private:
    void pull();
    Context* ctx_ = nullptr;
    pcg_me* me_ = nullptr;
    pcg_grid_params grid_{};
    std::vector<pcg_substrate_params> subs_;
    std::vector<float> mirror_, gx_, gy_, gz_;
    bool mirror_valid_ = false, mirror_dirty_ = false;
    friend class CellMechanics;
};

class CellMechanics {
public:
    CellMechanics() = default;
    ~CellMechanics();

    template <class Config>
    void initialize(const Config& config, Context* ctx, uint32_t max_cells = 200000);

    // clear/build/forces + integrate (cell_mechanics.mm:84-97)
    template <class Cells>
    void update(Cells& cells, float dt);
    // bin + sort + cell-start table + forces (cell_mechanics.mm:99-111)
    template <class Cells>
    void computeForces(Cells& cells, float dt);
    // AB2 + clamp (cell_mechanics.mm:113-120)
    template <class Cells>
    void integratePositions(Cells& cells, float dt);

    uint32_t totalMechVoxels() const { return total_; }
    const pcg_mechanics_params& params() const { return params_; }
    uint32_t voxelIndexFromPosition(float px, float py, float pz) const;   // cell_mechanics.h:40-50
    uint32_t voxelCellCount(uint32_t v) const;                             // cell_mechanics.h:53-56
    const uint32_t* voxelCells(uint32_t v) const;                          // cell_mechanics.h:59-62
    void syncHashPointers();                                               // cell_mechanics.mm:122-133

    pcg_cells* device_cells() const { return cells_; }
private:
    template <class Cells>
    void push(Cells& cells);
    template <class Cells>
    void pull(Cells& cells);
    Context* ctx_ = nullptr;
    pcg_mech* mech_ = nullptr;
    pcg_cells* cells_ = nullptr;
    pcg_mechanics_params params_{};
    float ox_ = 0, oy_ = 0, oz_ = 0;
    uint32_t total_ = 0, max_cells_ = 0, n_substrates_ = 0;
    std::vector<uint32_t> start_, sorted_;
};

// MotilityData (src/motility.h:20-66): the same members, indexed as the
// reference indexes its arrays, held in host vectors.  updateMotility keeps
// a device copy in step with them.
struct MotilityData {
    uint32_t max_cells = 0;
    uint32_t num_cells = 0;
    std::vector<double> persistence_time, motility_elapsed, motility_bias;
    std::vector<double> motility_vec_x, motility_vec_y, motility_vec_z;
    std::vector<uint32_t> is_motile, restrict_to_2D;
    std::vector<int32_t> chemotaxis_index, chemotaxis_direction;
    std::vector<double> chemotactic_sensitivity;   // [cell * n_substrates + s]
    uint32_t n_substrates = 0;
    // The reference draws from an unseeded generator.  Here draw k of cell i
    // in update number `step` is a counter-based uniform of (seed, i, step, k);
    // updateMotility advances step by one per call.
    uint64_t seed = 0;
    uint64_t step = 0;

    MotilityData() = default;
    ~MotilityData();
    MotilityData(const MotilityData&) = delete;
    MotilityData& operator=(const MotilityData&) = delete;

    void allocate(uint32_t max_cells);               // motility.cpp:90-107
    void allocateSubstrate(uint32_t n_substrates);   // motility.cpp:109-116
    void free_all();                                 // motility.cpp:118-131
    void setDefaults(uint32_t index);                // motility.cpp:133-152
    void swapRemove(uint32_t index, uint32_t last);  // motility.cpp:154-175

    // the device state for this context, made on first use and again after
    // allocate / allocateSubstrate change the sizes
    pcg_motility* device(Context* ctx);
private:
    friend class Context;
    void release();
    pcg_motility* dev_ = nullptr;
    Context* dev_ctx_ = nullptr;
};

// updateMotility(cells, mot, density, grid, dt) (motility.cpp:179-293): the
// density and grid are the Microenvironment's, read on the device.  Adds the
// motility vector of each living motile cell to its velocity and writes back
// motility_elapsed and motility_vec_*.  layout PCG_MOT_REFERENCE reads the
// gradient as the reference does (see include/pcg.h).
template <class Cells>
void updateMotility(Cells& cells, MotilityData& mot, Microenvironment& micro, double dt,
                    int layout = PCG_MOT_REFERENCE);

// writeMatlabSnapshots(cells, density, grid, frame, folder)
// (output_writer.cpp:295-452): output%08d_cells.mat and
// output%08d_microenvironment0.mat in output_folder, written before the call
// returns, byte-identical to the reference writer's files.
template <class Cells>
void writeMatlabSnapshots(const Cells& cells, Microenvironment& micro, int frame_index,
                          const std::string& output_folder);

// The asynchronous form: frame() builds the matrices on the device behind the
// work already queued and returns; a host thread writes the files while the
// simulation goes on.  wait() blocks until every queued file is written and
// throws for one that could not be.
class SnapshotWriter {
public:
    explicit SnapshotWriter(Context* ctx);
    ~SnapshotWriter();
    SnapshotWriter(const SnapshotWriter&) = delete;
    SnapshotWriter& operator=(const SnapshotWriter&) = delete;
    template <class Cells>
    void frame(const Cells& cells, Microenvironment& micro, int frame_index, const std::string& output_folder);
    void wait();
private:
    Context* ctx_ = nullptr;
    pcg_snapshot* snap_ = nullptr;
};

}  // namespace pcg

#include "pcg_host_impl.h"
