// sim_main.cpp — Linux twin of the reference's main-loop hot path
// (src/main.mm:275-415) built on the drop-in classes of pcg_host.h.
//
// Per diffusion step: simulateDiffusionDecay -> applyDirichletBC ->
// secretion of every live cell; every dt_mechanics: computeForces ->
// (motility would add to velocity here) -> integratePositions.  Phenotype,
// output and rules are outside the hot path and not run.
//
//   pcg_sim <cells.bin> <n_steps> <out.bin>
// cells.bin: uint32 n_cells, uint32 max_cells, float block[28 * max_cells],
//            then double secretion/uptake/saturation/net_export [n_cells] each
// out.bin:   float density[50 * 50], float block[28 * max_cells]
// The domain is the 2-D plain configuration: [-500, 500]^2, dx 20, one
// O2-like substrate (D 1e5, decay 0.1, Dirichlet 38, initial 38).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "pcg_host.h"

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s cells.bin n_steps out.bin\n", argv[0]);
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) {
        std::perror("cells.bin");
        return 2;
    }
    uint32_t n = 0, maxc = 0;
    if (std::fread(&n, 4, 1, f) != 1 || std::fread(&maxc, 4, 1, f) != 1 || n > maxc) {
        std::fprintf(stderr, "bad header\n");
        return 2;
    }
    pcg::SimConfig cfg;
    cfg.x_min = cfg.y_min = -500.0f;
    cfg.x_max = cfg.y_max = 500.0f;
    cfg.z_min = -10.0f;
    cfg.z_max = 10.0f;
    cfg.use_2D = true;
    cfg.grid.dx = cfg.grid.dy = cfg.grid.dz = 20.0f;
    cfg.dt_diffusion = 0.01f;
    cfg.dt_mechanics = 0.1f;
    pcg::SubstrateConfig o2;
    o2.name = "oxygen";
    o2.diffusion_coeff = 1e5f;
    o2.decay_rate = 0.1f;
    o2.initial_value = 38.0f;
    o2.dirichlet_enabled = true;
    o2.dirichlet_value = 38.0f;
    cfg.substrates.push_back(o2);

    pcg::CellStore cells(maxc, 1);
    cells.num_cells = n;
    bool ok = std::fread(cells.block.data(), 4, cells.block.size(), f) == cells.block.size();
    for (auto* v : {&cells.secretion_rate, &cells.uptake_rate, &cells.saturation_density, &cells.net_export_rate})
        ok = ok && std::fread(v->data(), 8, n, f) == n;
    std::fclose(f);
    if (!ok) {
        std::fprintf(stderr, "short read\n");
        return 2;
    }
    const int steps = std::atoi(argv[2]);
    try {
        pcg::Context ctx(0);
        pcg::Microenvironment microenv;
        microenv.initialize(cfg, &ctx);
        pcg::CellMechanics mechanics;
        mechanics.initialize(cfg, &ctx, maxc);
        double mech_acc = 0.0, t_diff = 0.0, t_mech = 0.0;
        int nd = 0, nm = 0;
        const double dt_d = cfg.dt_diffusion, dt_m = cfg.dt_mechanics;
        using clk = std::chrono::steady_clock;
        for (int s = 0; s < steps; ++s) {
            auto t0 = clk::now();
            microenv.simulateDiffusionDecay();
            microenv.applyDirichletBC();
            microenv.secreteAll(cells, dt_d);
            ctx.waitForCompletion();
            t_diff += std::chrono::duration<double>(clk::now() - t0).count();
            ++nd;
            mech_acc += dt_d;
            if (mech_acc >= dt_m - 0.5 * dt_d) {
                t0 = clk::now();
                mechanics.computeForces(cells, static_cast<float>(dt_m));
                mechanics.syncHashPointers();
                // updateMotility(...) would add to velocity here (main.mm:383-384)
                mechanics.integratePositions(cells, static_cast<float>(dt_m));
                ctx.waitForCompletion();
                t_mech += std::chrono::duration<double>(clk::now() - t0).count();
                ++nm;
                mech_acc = 0.0;
            }
        }
        std::printf("Diffusion (GPU): %.3f ms/step over %d steps\n", nd ? 1000.0 * t_diff / nd : 0.0, nd);
        std::printf("Mechanics (GPU): %.3f ms/step over %d steps\n", nm ? 1000.0 * t_mech / nm : 0.0, nm);
        std::printf("voxel 0 cells: %u, centre voxel count %u\n", mechanics.voxelCellCount(0),
                    mechanics.voxelCellCount(mechanics.voxelIndexFromPosition(0.f, 0.f, 0.f)));
        FILE* o = std::fopen(argv[3], "wb");
        if (!o) {
            std::perror("out.bin");
            return 2;
        }
        const float* d = microenv.densityBuffer();
        std::fwrite(d, 4, microenv.numVoxels(), o);
        std::fwrite(cells.block.data(), 4, cells.block.size(), o);
        std::fclose(o);
    } catch (const pcg::Error& e) {
        std::fprintf(stderr, "pcg error %d: %s\n", e.status, e.what());
        return 1;
    }
    return 0;
}
