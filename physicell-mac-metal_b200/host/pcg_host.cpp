// pcg_host.cpp — non-template members of the host drop-ins (see pcg_host.h).
#include "pcg_host.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <utility>

namespace pcg {

CellStore::CellStore(uint32_t maxc, uint32_t S) : max_cells(maxc), n_substrates(S)
{
    block.assign(static_cast<size_t>(PCG_NUM_FIELDS) * max_cells, 0.0f);
    position_x = block.data();
    const size_t n = static_cast<size_t>(max_cells) * S;
    secretion_rate.assign(n, 0.0);
    uptake_rate.assign(n, 0.0);
    saturation_density.assign(n, 0.0);
    net_export_rate.assign(n, 0.0);
    current_death_model.assign(max_cells, 0);
}

uint32_t CellStore::addCell()
{
    if (num_cells >= max_cells) return UINT32_MAX;   // cell_data.cpp:398-401
    return num_cells++;
}

Context::Context(int device)
{
    const int st = pcg_create(device, &ctx_);
    if (st != PCG_OK) throw Error(st, std::string("pcg_create: ") + pcg_last_error_string(nullptr));
}

void release_stores(const Context* ctx);

Context::~Context()
{
    while (!motility_.empty()) motility_.back()->release();   // release() unregisters
    release_stores(this);
    pcg_destroy(ctx_);
}

void Context::waitForCompletion() { check(pcg_sync(ctx_)); }

void Context::check(int status) const
{
    if (status != PCG_OK) throw Error(status, pcg_last_error_string(ctx_));
}

namespace {
std::mutex g_store_mu;
std::map<std::pair<const void*, const void*>, pcg_cells*> g_stores;
}  // namespace

pcg_cells* device_store(Context* ctx, const void* host_block, uint32_t max_cells, uint32_t n_substrates)
{
    std::lock_guard<std::mutex> lk(g_store_mu);
    auto key = std::make_pair(static_cast<const void*>(ctx), host_block);
    auto it = g_stores.find(key);
    if (it != g_stores.end()) return it->second;
    pcg_cells* c = nullptr;
    ctx->check(pcg_cells_create(ctx->get(), max_cells, n_substrates, &c));
    g_stores[key] = c;
    return c;
}

void release_stores(const Context* ctx)
{
    std::lock_guard<std::mutex> lk(g_store_mu);
    for (auto it = g_stores.begin(); it != g_stores.end();) {
        if (it->first.first == ctx) {
            pcg_cells_destroy(it->second);
            it = g_stores.erase(it);
        } else {
            ++it;
        }
    }
}

// ------------------------------------------------------------------ Microenvironment

Microenvironment::~Microenvironment() { pcg_me_destroy(me_); }

void Microenvironment::push_host_writes()
{
    if (mirror_dirty_) {
        ctx_->check(pcg_me_upload(me_, mirror_.data(), mirror_.size()));
        mirror_dirty_ = false;
    }
}

void Microenvironment::pull()
{
    if (!mirror_valid_) {
        ctx_->check(pcg_me_download(me_, mirror_.data(), mirror_.size()));
        mirror_valid_ = true;
    }
}

void Microenvironment::simulateDiffusionDecay()
{
    push_host_writes();
    ctx_->check(pcg_me_diffuse(me_, 1));
    mirror_valid_ = false;
}

void Microenvironment::applyDirichletBC()
{
    push_host_writes();
    ctx_->check(pcg_me_apply_dirichlet(me_));
    mirror_valid_ = false;
}

float* Microenvironment::densityBuffer()
{
    pull();
    mirror_dirty_ = true;   // the caller may write through the pointer
    return mirror_.data();
}

float Microenvironment::getDensity(uint32_t v, uint32_t s) const
{
    const_cast<Microenvironment*>(this)->pull();
    return mirror_[static_cast<size_t>(s) * numVoxels() + v];
}

void Microenvironment::setDensity(uint32_t v, uint32_t s, float value)
{
    pull();
    mirror_[static_cast<size_t>(s) * numVoxels() + v] = value;
    mirror_dirty_ = true;
}

void Microenvironment::applySecretion(uint32_t v, uint32_t s, float sec, float upt, float sat, float dt)
{
    pull();
    float& rho = mirror_[static_cast<size_t>(s) * numVoxels() + v];
    const float denom = 1.0f + dt * (sec + upt);
    rho = (rho + dt * sec * sat) / denom;
    mirror_dirty_ = true;
}

uint32_t Microenvironment::voxelIndex(float x, float y, float z) const
{
    int i = static_cast<int>((x - grid_.x_min) / grid_.dx);
    int j = static_cast<int>((y - grid_.y_min) / grid_.dy);
    int k = static_cast<int>((z - grid_.z_min) / grid_.dz);
    i = i < 0 ? 0 : (i >= static_cast<int>(grid_.nx) ? static_cast<int>(grid_.nx) - 1 : i);
    j = j < 0 ? 0 : (j >= static_cast<int>(grid_.ny) ? static_cast<int>(grid_.ny) - 1 : j);
    k = k < 0 ? 0 : (k >= static_cast<int>(grid_.nz) ? static_cast<int>(grid_.nz) - 1 : k);
    return static_cast<uint32_t>(k) * grid_.nx * grid_.ny + static_cast<uint32_t>(j) * grid_.nx +
           static_cast<uint32_t>(i);
}

void Microenvironment::computeGradients()
{
    push_host_writes();
    const size_t n = mirror_.size();
    gx_.resize(n);
    gy_.resize(n);
    gz_.resize(n);
    ctx_->check(pcg_me_gradients(me_, gx_.data(), gy_.data(), gz_.data(), n));
}

void Microenvironment::getGradient(uint32_t v, uint32_t s, float& gx, float& gy, float& gz) const
{
    const size_t i = static_cast<size_t>(s) * numVoxels() + v;
    gx = i < gx_.size() ? gx_[i] : 0.0f;
    gy = i < gy_.size() ? gy_[i] : 0.0f;
    gz = i < gz_.size() ? gz_[i] : 0.0f;
}

// ------------------------------------------------------------------ CellMechanics

CellMechanics::~CellMechanics() { pcg_mech_destroy(mech_); }

uint32_t CellMechanics::voxelIndexFromPosition(float px, float py, float pz) const
{
    int vi = static_cast<int>((px - ox_) / params_.mechanics_voxel_size);
    int vj = static_cast<int>((py - oy_) / params_.mechanics_voxel_size);
    int vk = static_cast<int>((pz - oz_) / params_.mechanics_voxel_size);
    vi = std::max(0, std::min(vi, static_cast<int>(params_.mech_grid_nx) - 1));
    vj = std::max(0, std::min(vj, static_cast<int>(params_.mech_grid_ny) - 1));
    vk = std::max(0, std::min(vk, static_cast<int>(params_.mech_grid_nz) - 1));
    return static_cast<uint32_t>(vk) * params_.mech_grid_ny * params_.mech_grid_nx +
           static_cast<uint32_t>(vj) * params_.mech_grid_nx + static_cast<uint32_t>(vi);
}

void CellMechanics::syncHashPointers()
{
    start_.assign(static_cast<size_t>(total_) + 1, 0);
    sorted_.assign(std::max<uint32_t>(max_cells_, 1), 0);
    ctx_->check(pcg_mech_bins(mech_, start_.data(), sorted_.data()));
}

uint32_t CellMechanics::voxelCellCount(uint32_t v) const
{
    if (start_.empty() || v >= total_) return 0;
    return start_[v + 1] - start_[v];
}

const uint32_t* CellMechanics::voxelCells(uint32_t v) const
{
    if (start_.empty() || v >= total_) return nullptr;
    return sorted_.data() + start_[v];
}

// ------------------------------------------------------------------ MotilityData

MotilityData::~MotilityData() { release(); }

void MotilityData::release()
{
    if (!dev_) return;
    pcg_motility_destroy(dev_);
    auto& reg = dev_ctx_->motility_;
    reg.erase(std::remove(reg.begin(), reg.end(), this), reg.end());
    dev_ = nullptr;
    dev_ctx_ = nullptr;
}

void MotilityData::allocate(uint32_t max_c)
{
    release();
    max_cells = max_c;
    num_cells = 0;
    n_substrates = 0;
    for (auto* v : {&persistence_time, &motility_elapsed, &motility_bias, &motility_vec_x, &motility_vec_y,
                    &motility_vec_z})
        v->assign(max_c, 0.0);
    is_motile.assign(max_c, 0);
    restrict_to_2D.assign(max_c, 0);
    chemotaxis_index.assign(max_c, 0);
    chemotaxis_direction.assign(max_c, 0);
    chemotactic_sensitivity.clear();
}

void MotilityData::allocateSubstrate(uint32_t nsubs)
{
    release();
    n_substrates = nsubs;
    chemotactic_sensitivity.assign(static_cast<size_t>(max_cells) * nsubs, 0.0);
}

void MotilityData::free_all()
{
    release();
    for (auto* v : {&persistence_time, &motility_elapsed, &motility_bias, &motility_vec_x, &motility_vec_y,
                    &motility_vec_z, &chemotactic_sensitivity})
        v->clear();
    is_motile.clear();
    restrict_to_2D.clear();
    chemotaxis_index.clear();
    chemotaxis_direction.clear();
    n_substrates = 0;
}

void MotilityData::setDefaults(uint32_t i)
{
    if (i >= max_cells) throw Error(PCG_ERR_INVALID, "MotilityData::setDefaults: index out of range");
    // PhysiCell's defaults: 15 min persistence, bias 0.5, not motile, 2-D,
    // chemotaxis up the first substrate, no per-substrate sensitivity
    persistence_time[i] = 15.0;
    motility_elapsed[i] = 0.0;
    motility_bias[i] = 0.5;
    motility_vec_x[i] = motility_vec_y[i] = motility_vec_z[i] = 0.0;
    is_motile[i] = 0;
    restrict_to_2D[i] = 1;
    chemotaxis_index[i] = 0;
    chemotaxis_direction[i] = 1;
    if (n_substrates)
        std::fill_n(chemotactic_sensitivity.begin() + static_cast<size_t>(i) * n_substrates, n_substrates, 0.0);
}

void MotilityData::swapRemove(uint32_t i, uint32_t last)
{
    if (i == last) return;
    for (auto* v : {&persistence_time, &motility_elapsed, &motility_bias, &motility_vec_x, &motility_vec_y,
                    &motility_vec_z})
        (*v)[i] = (*v)[last];
    is_motile[i] = is_motile[last];
    restrict_to_2D[i] = restrict_to_2D[last];
    chemotaxis_index[i] = chemotaxis_index[last];
    chemotaxis_direction[i] = chemotaxis_direction[last];
    if (n_substrates)
        std::copy_n(chemotactic_sensitivity.begin() + static_cast<size_t>(last) * n_substrates, n_substrates,
                    chemotactic_sensitivity.begin() + static_cast<size_t>(i) * n_substrates);
}

pcg_motility* MotilityData::device(Context* ctx)
{
    if (dev_ && dev_ctx_ != ctx) release();
    if (!dev_) {
        ctx->check(pcg_motility_create(ctx->get(), max_cells, n_substrates, &dev_));
        dev_ctx_ = ctx;
        ctx->motility_.push_back(this);
    }
    return dev_;
}

// ------------------------------------------------------------------ SnapshotWriter

SnapshotWriter::SnapshotWriter(Context* ctx) : ctx_(ctx)
{
    ctx_->check(pcg_snapshot_create(ctx_->get(), &snap_));
}

SnapshotWriter::~SnapshotWriter() { pcg_snapshot_destroy(snap_); }

void SnapshotWriter::wait() { ctx_->check(pcg_snapshot_wait(snap_)); }

}  // namespace pcg
