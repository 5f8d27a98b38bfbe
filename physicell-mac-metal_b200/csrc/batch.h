// batch.h — the batch engine (shared by pcg_batch and the server).
#pragma once

#include <string>
#include <vector>

#include "runtime.h"

namespace pcg {

uint64_t instance_bytes(const pcg_instance_desc& d);

class Batch;

// Device state to start an instance from (serving: a request that keeps
// running when the batch is rebuilt moves device-to-device).
struct DevSource {
    const Batch* batch = nullptr;
    uint32_t index = 0;
};

class Batch {
public:
    pcg_ctx* ctx = nullptr;
    Diffusion d;
    Cells c_;
    Mechanics m_;
    std::vector<uint32_t> ncell;
    double dt_diff = 0.0, dt_mech = 0.0, accum = 0.0;
    bool use_graphs = true, profile = false, any_refresh = false;
    std::string tune_cache;
    cudaGraphExec_t g_diff = nullptr, g_mech = nullptr;
    uint64_t launches_diff = 0, launches_mech = 0;
    // A whole mechanics period (the sub-steps from a reset accumulator to
    // the one that fires, mechanics included) as one graph: period_len
    // sub-steps per launch where a call covers them, single sub-step
    // graphs elsewhere.
    static constexpr int kMaxPeriod = 64;   // longer periods run as single sub-steps
    cudaGraphExec_t g_period = nullptr;
    uint64_t launches_period = 0;
    int period_len = 0;
    cudaEvent_t ev[8] = {};
    // Staging of the whole-batch transfers (made on first use): host copies
    // run on the context's copy streams, device-to-device copies on its
    // stream; *_done / in_used mark when a staging buffer may be reused.
    DevBuf stage_in, stage_cells, stage_dens;
    cudaEvent_t ev_in_done = nullptr, ev_in_used = nullptr, ev_cells_ready = nullptr, ev_cells_done = nullptr,
                ev_dens_ready = nullptr, ev_dens_done = nullptr;
    double phase_ms[PCG_N_PHASES] = {};
    uint64_t sweep_steps = 0, diff_steps = 0, mech_steps = 0;

    Batch() = default;
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;
    ~Batch();

    // src (optional, one entry per instance, batch == nullptr for none)
    // takes the instance's state from another batch; masked = the step
    // kernels read a per-instance step mask (set by step_masked).
    int create(pcg_ctx* c, const pcg_instance_desc* descs, uint32_t n, const pcg_batch_options* opt,
               const std::vector<DevSource>* src = nullptr, bool masked = false);
    // n_steps main-loop sub-steps (mechanics when the accumulator fires)
    int step(int n_steps);
    // One sub-step with host-computed per-instance bits (STEP_DIFFUSE /
    // STEP_MECH) from 'mask_host' (pinned, n_instances bytes, must stay
    // unchanged until the stream reaches this step).
    int step_masked(const uint8_t* mask_host, bool any_mech);
    DevBuf mask_d;
    bool masked = false;
    // One sub-step for the instances whose mask bits are set (mask on the device).
    int run_step(bool mech, bool timed, const uint8_t* mask);
    uint64_t count_launches(bool mech) const;
    std::string describe() const;
    // Neighbour-set diagnostics of the force pass (the mechanics graph is
    // captured again with them).
    int set_diagnostics(bool on);

private:
    int capture(bool mech, cudaGraphExec_t* out, uint64_t* launches, int n_diff = 0);
    // Launch shapes of the cell kernels: pinned by the options, else cached
    // by shape bucket or measured on the batch's own data (the state the
    // timed launches write is saved first and put back).
    int tune_cells(const pcg_batch_options* opt, bool tune);
};

}  // namespace pcg
