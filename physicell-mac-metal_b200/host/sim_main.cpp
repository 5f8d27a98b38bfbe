// sim_main.cpp — Linux twin of the reference's main-loop hot path
// (src/main.mm:275-415) built on the drop-in classes of pcg_host.h.
//
// Per diffusion step: simulateDiffusionDecay -> applyDirichletBC ->
// secretion of every live cell; every dt_mechanics: computeForces ->
// updateMotility (with --motility) -> integratePositions.  With --mat, the
// .mat frames of main.mm:299 (frame 0, before the loop, asynchronous) and
// main.mm:424 (frame 1, after it) are written.  Phenotype, the other writers
// and rules are outside the hot path and not run.
//
//   pcg_sim <cells.bin> <n_steps> <out.bin> [--motility mot.bin --seed N] [--mat DIR]
// cells.bin: uint32 n_cells, uint32 max_cells, float block[28 * max_cells],
//            then double secretion/uptake/saturation/net_export [n_cells] each
// mot.bin:   double persistence_time, elapsed, bias, vec_x, vec_y, vec_z [n_cells]
//            each, uint32 is_motile, restrict_to_2D, int32 chemotaxis_index,
//            chemotaxis_direction [n_cells] each, uint32 n_sens, then double
//            sensitivity [n_cells * n_sens] (cell-major)
// out.bin:   float density[50 * 50], float block[28 * max_cells]; with
//            --motility then double elapsed [n_cells], vec [3 * n_cells]
// The domain is the 2-D plain configuration: [-500, 500]^2, dx 20, one
// O2-like substrate (D 1e5, decay 0.1, Dirichlet 38, initial 38).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pcg_host.h"

namespace {

template <class T>
bool read_n(FILE* f, std::vector<T>& v, size_t n)
{
    v.resize(n);
    return std::fread(v.data(), sizeof(T), n, f) == n;
}

bool read_motility(const char* path, uint32_t n, uint32_t max_cells, pcg::MotilityData& mot)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    mot.allocate(max_cells);
    std::vector<double> d;
    std::vector<uint32_t> u;
    std::vector<int32_t> k;
    bool ok = true;
    for (auto* dst : {&mot.persistence_time, &mot.motility_elapsed, &mot.motility_bias, &mot.motility_vec_x,
                      &mot.motility_vec_y, &mot.motility_vec_z}) {
        ok = ok && read_n(f, d, n);
        if (ok) std::copy(d.begin(), d.end(), dst->begin());
    }
    for (auto* dst : {&mot.is_motile, &mot.restrict_to_2D}) {
        ok = ok && read_n(f, u, n);
        if (ok) std::copy(u.begin(), u.end(), dst->begin());
    }
    for (auto* dst : {&mot.chemotaxis_index, &mot.chemotaxis_direction}) {
        ok = ok && read_n(f, k, n);
        if (ok) std::copy(k.begin(), k.end(), dst->begin());
    }
    uint32_t n_sens = 0;
    ok = ok && std::fread(&n_sens, 4, 1, f) == 1;
    if (ok && n_sens) {
        mot.allocateSubstrate(n_sens);
        ok = read_n(f, d, static_cast<size_t>(n) * n_sens);
        if (ok) std::copy(d.begin(), d.end(), mot.chemotactic_sensitivity.begin());
    }
    std::fclose(f);
    mot.num_cells = n;
    return ok;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s cells.bin n_steps out.bin [--motility mot.bin --seed N] [--mat DIR]\n",
                     argv[0]);
        return 2;
    }
    const char* mot_path = nullptr;
    const char* mat_dir = nullptr;
    uint64_t seed = 0;
    for (int a = 4; a < argc; ++a) {
        if (!std::strcmp(argv[a], "--motility") && a + 1 < argc) mot_path = argv[++a];
        else if (!std::strcmp(argv[a], "--seed") && a + 1 < argc) seed = std::strtoull(argv[++a], nullptr, 10);
        else if (!std::strcmp(argv[a], "--mat") && a + 1 < argc) mat_dir = argv[++a];
        else {
            std::fprintf(stderr, "unknown argument %s\n", argv[a]);
            return 2;
        }
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
    pcg::MotilityData motility;
    if (mot_path && !read_motility(mot_path, n, maxc, motility)) {
        std::fprintf(stderr, "bad motility file\n");
        return 2;
    }
    motility.seed = seed;
    const int steps = std::atoi(argv[2]);
    try {
        pcg::Context ctx(0);
        pcg::Microenvironment microenv;
        microenv.initialize(cfg, &ctx);
        pcg::CellMechanics mechanics;
        mechanics.initialize(cfg, &ctx, maxc);
        pcg::SnapshotWriter snapshots(&ctx);
        if (mat_dir) snapshots.frame(cells, microenv, 0, mat_dir);   // written while the loop runs
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
                if (mot_path) pcg::updateMotility(cells, motility, microenv, dt_m);
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
        if (mat_dir) {
            snapshots.wait();
            pcg::writeMatlabSnapshots(cells, microenv, 1, mat_dir);
        }
        FILE* o = std::fopen(argv[3], "wb");
        if (!o) {
            std::perror("out.bin");
            return 2;
        }
        const float* d = microenv.densityBuffer();
        std::fwrite(d, 4, microenv.numVoxels(), o);
        std::fwrite(cells.block.data(), 4, cells.block.size(), o);
        if (mot_path) {
            std::fwrite(motility.motility_elapsed.data(), 8, n, o);
            for (auto* v : {&motility.motility_vec_x, &motility.motility_vec_y, &motility.motility_vec_z})
                std::fwrite(v->data(), 8, n, o);
        }
        std::fclose(o);
    } catch (const pcg::Error& e) {
        std::fprintf(stderr, "pcg error %d: %s\n", e.status, e.what());
        return 1;
    }
    return 0;
}
