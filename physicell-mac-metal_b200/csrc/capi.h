// capi.h — the single-simulation objects behind the C ABI (shared by the
// files that implement its entry points).
#pragma once

#include "runtime.h"

struct pcg_me {
    pcg_ctx* ctx = nullptr;
    pcg::Diffusion d;
};

struct pcg_cells {
    pcg_ctx* ctx = nullptr;
    pcg::Cells c;
    uint32_t S = 0;
    const pcg_me* bound_me = nullptr;
    const pcg_mech* bound_mech = nullptr;
};

struct pcg_mech {
    pcg_ctx* ctx = nullptr;
    pcg::Mechanics m;
    pcg_mechanics_params p{};
    float ox = 0, oy = 0, oz = 0;
};
