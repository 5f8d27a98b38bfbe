// pcg_host_impl.h — template members of the host drop-ins (included by pcg_host.h).
#pragma once

#include <algorithm>
#include <cstring>

namespace pcg {

// Device cell store shared by Microenvironment and CellMechanics for one
// host cell block (the reference shares the CellData GPU block the same way).
pcg_cells* device_store(Context* ctx, const void* host_block, uint32_t max_cells, uint32_t n_substrates);

template <class Cells>
inline const float* block_of(const Cells& c) { return c.position_x; }

template <class Config>
void Microenvironment::initialize(const Config& config, Context* ctx)
{
    ctx_ = ctx;
    // microenvironment.mm:33-35: truncating voxel counts, nz = 1 in 2-D
    grid_ = pcg_grid_params{};
    grid_.nx = static_cast<uint32_t>((config.x_max - config.x_min) / config.grid.dx);
    grid_.ny = static_cast<uint32_t>((config.y_max - config.y_min) / config.grid.dy);
    grid_.nz = config.use_2D ? 1u : static_cast<uint32_t>((config.z_max - config.z_min) / config.grid.dz);
    grid_.dx = config.grid.dx;
    grid_.dy = config.grid.dy;
    grid_.dz = config.grid.dz;
    grid_.x_min = config.x_min;
    grid_.y_min = config.y_min;
    grid_.z_min = config.z_min;
    grid_.dt = config.dt_diffusion;
    grid_.n_substrates = static_cast<uint32_t>(config.substrates.size());
    subs_.assign(grid_.n_substrates, pcg_substrate_params{});
    std::vector<float> init(grid_.n_substrates);
    for (uint32_t s = 0; s < grid_.n_substrates; ++s) {
        subs_[s].diffusion_coefficient = config.substrates[s].diffusion_coeff;
        subs_[s].decay_rate = config.substrates[s].decay_rate;
        subs_[s].supply_rate = 0.0f;
        subs_[s].target_value = config.substrates[s].dirichlet_value;
        subs_[s].dirichlet_enabled = config.substrates[s].dirichlet_enabled ? 1u : 0u;
        init[s] = config.substrates[s].initial_value;
    }
    ctx_->check(pcg_me_create(ctx_->get(), &grid_, subs_.data(), &me_));
    if (grid_.n_substrates) ctx_->check(pcg_me_fill(me_, init.data()));
    mirror_.assign(static_cast<size_t>(numVoxels()) * grid_.n_substrates, 0.0f);
    mirror_valid_ = mirror_dirty_ = false;
}

// The CPU owns the cell block: refresh the device copy of the 28 fields and,
// with rates, of the per-substrate secretion rates and the live mask.
template <class Cells>
pcg_cells* sync_cells(Context* ctx, const Cells& cells, uint32_t n_substrates, bool rates)
{
    pcg_cells* dc = device_store(ctx, block_of(cells), cells.max_cells, n_substrates);
    ctx->check(pcg_cells_upload(dc, block_of(cells), cells.num_cells, cells.max_cells));
    if (rates) {
        std::vector<uint8_t> active(cells.num_cells, 1);
        for (uint32_t i = 0; i < cells.num_cells && i < cells.current_death_model.size(); ++i)
            active[i] = cells.current_death_model[i] == 0 ? 1 : 0;   // main.mm:360
        ctx->check(pcg_cells_set_secretion(dc, cells.secretion_rate.data(), cells.uptake_rate.data(),
                                           cells.saturation_density.data(), cells.net_export_rate.data(),
                                           active.data()));
    }
    return dc;
}

template <class Cells>
void Microenvironment::secreteAll(Cells& cells, double dt)
{
    push_host_writes();
    pcg_cells* dc = sync_cells(ctx_, cells, grid_.n_substrates, true);
    ctx_->check(pcg_me_secrete(me_, dc, dt));
    mirror_valid_ = false;
}

template <class Cells>
void Microenvironment::step(Cells& cells)
{
    simulateDiffusionDecay();
    applyDirichletBC();
    secreteAll(cells, static_cast<double>(grid_.dt));
}

template <class Config>
void CellMechanics::initialize(const Config& config, Context* ctx, uint32_t max_cells)
{
    ctx_ = ctx;
    // cell_mechanics.mm:26-41
    const float vs = 30.0f;
    params_ = pcg_mechanics_params{};
    params_.dt = config.dt_mechanics;
    params_.cell_cell_repulsion = 10.0f;
    params_.cell_cell_adhesion = 0.4f;
    params_.max_interaction_distance = vs;
    params_.mechanics_voxel_size = vs;
    params_.mech_grid_nx = std::max(1u, static_cast<uint32_t>((config.x_max - config.x_min) / vs));
    params_.mech_grid_ny = std::max(1u, static_cast<uint32_t>((config.y_max - config.y_min) / vs));
    params_.mech_grid_nz = config.use_2D ? 1u : std::max(1u, static_cast<uint32_t>((config.z_max - config.z_min) / vs));
    total_ = params_.mech_grid_nx * params_.mech_grid_ny * params_.mech_grid_nz;
    ox_ = config.x_min;
    oy_ = config.y_min;
    oz_ = config.z_min;
    max_cells_ = max_cells;
    n_substrates_ = static_cast<uint32_t>(config.substrates.size());
    ctx_->check(pcg_mech_create(ctx_->get(), &params_, ox_, oy_, oz_, max_cells_, &mech_));
}

template <class Cells>
void CellMechanics::push(Cells& cells)
{
    cells_ = device_store(ctx_, block_of(cells), cells.max_cells, n_substrates_);
    ctx_->check(pcg_cells_upload(cells_, block_of(cells), cells.num_cells, cells.max_cells));
}

template <class Cells>
void CellMechanics::pull(Cells& cells)
{
    ctx_->check(pcg_cells_download(cells_, const_cast<float*>(block_of(cells)), cells.max_cells));
}

template <class Cells>
void CellMechanics::computeForces(Cells& cells, float)
{
    if (cells.num_cells == 0) return;
    push(cells);
    ctx_->check(pcg_mech_forces(mech_, cells_));
    pull(cells);
}

template <class Cells>
void CellMechanics::integratePositions(Cells& cells, float dt)
{
    if (cells.num_cells == 0) return;
    push(cells);
    ctx_->check(pcg_mech_integrate(mech_, cells_, dt));
    pull(cells);
}

template <class Cells>
void CellMechanics::update(Cells& cells, float dt)
{
    if (cells.num_cells == 0) return;
    push(cells);
    ctx_->check(pcg_mech_update(mech_, cells_, dt));
    pull(cells);
}

template <class Cells>
void updateMotility(Cells& cells, MotilityData& mot, Microenvironment& micro, double dt, int layout)
{
    const uint32_t n = cells.num_cells;
    if (n == 0) return;
    if (n > mot.max_cells) throw Error(PCG_ERR_INVALID, "updateMotility: more cells than MotilityData::allocate'd");
    Context* ctx = micro.context();
    micro.push_host_writes();
    mot.num_cells = n;
    pcg_motility* dm = mot.device(ctx);
    std::vector<double> vec(3 * static_cast<size_t>(n));
    std::copy_n(mot.motility_vec_x.begin(), n, vec.begin());
    std::copy_n(mot.motility_vec_y.begin(), n, vec.begin() + n);
    std::copy_n(mot.motility_vec_z.begin(), n, vec.begin() + 2 * static_cast<size_t>(n));
    ctx->check(pcg_motility_upload(dm, n, mot.persistence_time.data(), mot.motility_elapsed.data(),
                                   mot.motility_bias.data(), vec.data(), mot.is_motile.data(),
                                   mot.restrict_to_2D.data(), mot.chemotaxis_index.data(),
                                   mot.chemotaxis_direction.data(),
                                   mot.n_substrates ? mot.chemotactic_sensitivity.data() : nullptr));
    pcg_cells* dc = sync_cells(ctx, cells, micro.getGridParams().n_substrates, false);
    ctx->check(pcg_motility_update(dm, dc, micro.handle(), dt, mot.seed, mot.step, layout));
    ++mot.step;
    ctx->check(pcg_motility_download(dm, mot.motility_elapsed.data(), vec.data()));
    std::copy_n(vec.begin(), n, mot.motility_vec_x.begin());
    std::copy_n(vec.begin() + n, n, mot.motility_vec_y.begin());
    std::copy_n(vec.begin() + 2 * static_cast<size_t>(n), n, mot.motility_vec_z.begin());
    ctx->check(pcg_cells_download(dc, const_cast<float*>(block_of(cells)), cells.max_cells));
}

template <class Cells>
uint32_t cell_types_of(const Cells& cells) { return cells.num_cell_types; }

template <class Cells>
void SnapshotWriter::frame(const Cells& cells, Microenvironment& micro, int frame_index,
                           const std::string& output_folder)
{
    micro.push_host_writes();
    pcg_cells* dc = sync_cells(ctx_, cells, micro.getGridParams().n_substrates, true);
    ctx_->check(pcg_snapshot_frame(snap_, micro.handle(), dc, cell_types_of(cells), output_folder.c_str(),
                                   frame_index));
}

template <class Cells>
void writeMatlabSnapshots(const Cells& cells, Microenvironment& micro, int frame_index,
                          const std::string& output_folder)
{
    SnapshotWriter w(micro.context());
    w.frame(cells, micro, frame_index, output_folder);
    w.wait();
}

}  // namespace pcg
