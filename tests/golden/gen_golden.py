"""Generate golden vectors by running the reference's own code on the CPU.

Needs oracle/_ref/libpcg_ref.so, which oracle/Makefile builds from the
reference tree (its Metal shader bodies compiled as C++ through
oracle/ref/metal_shim.h, and its processSecretion from
src/cell_phenotype.cpp).  Run from the repository root:

    python tests/golden/gen_golden.py

Writes tests/golden/*.npz: the seeded inputs and the reference's outputs.
The oracle tests check the oracle against these files, so the pin travels
without the reference tree.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle as po  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# (name, nx, ny, substrates [(D, decay, dirichlet, target)], steps, seed)
DIFFUSION_CASES = [
    ("diff_50x50_o2", 50, 50, [(1e5, 0.1, True, 38.0)], 3, 11),
    ("diff_16x16_two", 16, 16, [(0.0, 0.1, False, 0.0), (1e3, 0.5, True, 5.0)], 4, 12),
    ("diff_8x12_nodir", 8, 12, [(2.5e4, 0.2, False, 0.0)], 5, 13),
    ("diff_3x7", 3, 7, [(1e5, 0.1, True, 38.0)], 2, 14),
    ("diff_4x5", 4, 5, [(1e5, 0.1, True, 38.0), (3e3, 0.0, False, 1.0)], 2, 15),
    ("diff_2x9", 2, 9, [(1e5, 0.1, True, 38.0)], 2, 16),
    ("diff_33x17", 33, 17, [(7e4, 0.3, True, 10.0)], 3, 17),
    ("diff_uniform_T", 12, 10, [(1e5, 0.1, True, 38.0)], 3, 18),
]


def gen_diffusion():
    for name, nx, ny, subs_p, steps, seed in DIFFUSION_CASES:
        rng = np.random.default_rng(seed)
        S = len(subs_p)
        g = po.make_grid(nx, ny, 1, S, dx=20.0, dt=0.01, x_min=-0.5 * nx * 20, y_min=-0.5 * ny * 20)
        subs = po.make_subs(subs_p)
        if name == "diff_uniform_T":
            d0 = np.full(S * nx * ny, 38.0, np.float32)
        else:
            d0 = rng.uniform(0.0, 40.0, S * nx * ny).astype(np.float32)
        d = d0.copy()
        outs = []
        for _ in range(steps):
            po.ref_sweeps(d, g, subs)
            po.ref_dirichlet(d, g, subs)
            outs.append(d.copy())
        np.savez_compressed(os.path.join(OUT, name + ".npz"), nx=nx, ny=ny, subs=np.array(subs_p, np.float64),
                            steps=steps, density0=d0, density_steps=np.stack(outs))


def gen_secretion():
    rng = np.random.default_rng(21)
    nx, ny, S, n = 10, 10, 2, 300
    g = po.make_grid(nx, ny, 1, S, dx=20.0, dt=0.01)
    vox = rng.integers(0, nx * ny + 5, n).astype(np.uint32)      # a few out of range
    vox[:40] = 7                                                  # a crowded voxel
    vol = rng.uniform(1000, 4000, n).astype(np.float32)
    sec = rng.uniform(0, 10, n * S)
    upt = rng.uniform(0, 10, n * S)
    sat = rng.uniform(0, 40, n * S)
    ne = rng.uniform(-50, 50, n * S)
    d0 = rng.uniform(0, 40, S * nx * ny).astype(np.float32)
    d = d0.copy()
    po.ref_secretion(d, g, vox, vol, sec, upt, sat, ne, 0.01)
    np.savez_compressed(os.path.join(OUT, "secretion.npz"), nx=nx, ny=ny, S=S, voxel=vox, volume=vol, sec=sec,
                        upt=upt, sat=sat, ne=ne, density0=d0, density1=d)


def disc_cells(n, r, rng, max_cells, radius=8.41):
    soa = np.zeros(28 * max_cells, np.float32)
    rr = r * np.sqrt(rng.random(n))
    th = rng.random(n) * 2 * np.pi
    soa[0 * max_cells:0 * max_cells + n] = rr * np.cos(th)
    soa[1 * max_cells:1 * max_cells + n] = rr * np.sin(th)
    soa[9 * max_cells:9 * max_cells + n] = radius
    soa[11 * max_cells:11 * max_cells + n] = 2494.0
    soa[13 * max_cells:13 * max_cells + n] = 10.0
    soa[14 * max_cells:14 * max_cells + n] = 0.4
    soa[15 * max_cells:15 * max_cells + n] = 1.25
    return soa


def gen_mechanics():
    rng = np.random.default_rng(31)
    mc = 600
    n = 500
    m = po.mech_params(-500, 500, -500, 500, -10, 10, True, 0.1)
    origin = (-500.0, -500.0, -10.0)
    soa0 = disc_cells(n, 200.0, rng, mc)
    soa0[3 * mc:3 * mc + n] = rng.normal(0, 1, n)       # previous-step velocities for AB2
    soa0[6 * mc:6 * mc + n] = rng.normal(0, 1, n)
    s = soa0.copy()
    counts, cells = po.ref_forces(s, mc, n, m, origin)
    forces = s.copy()
    po.ref_integrate(s, mc, n, m, origin, 0.1)
    np.savez_compressed(os.path.join(OUT, "mechanics_2d.npz"), max_cells=mc, n=n, soa0=soa0, hash_counts=counts,
                        hash_cells=cells, soa_forces=forces, soa_integrated=s,
                        mech=np.array([m.mech_grid_nx, m.mech_grid_ny, m.mech_grid_nz], np.uint32))


def motility_case(rng, two_d, S, multi, n=300, mc=320):
    """Inputs for updateMotility where the result does not depend on the
    reference's unseeded draws: bias 1, persistence below dt."""
    nx, ny, nz = 20, 16, (1 if two_d else 12)
    grid = np.array([nx, ny, nz, S], np.uint32)
    geo = np.array([20.0, 20.0, 20.0, 0.01, -200.0, -160.0, -10.0 if two_d else -120.0], np.float32)
    dens = rng.uniform(0, 40, nx * ny * nz * S).astype(np.float32)
    soa = np.zeros(28 * mc, np.float32)
    soa[0:n] = rng.uniform(-210, 210, n)
    soa[mc:mc + n] = rng.uniform(-170, 170, n)
    soa[2 * mc:2 * mc + n] = 0 if two_d else rng.uniform(-130, 130, n)
    soa[3 * mc:6 * mc] = rng.normal(0, 1, 3 * mc)
    soa[16 * mc:16 * mc + n] = rng.uniform(0.5, 2, n)
    soa[25 * mc:25 * mc + n] = np.where(rng.random(n) < 0.9, 1, 0).astype(np.uint32).view(np.float32)
    st = po.motility_state(n, S if multi else 0)
    st["is_motile"][:] = rng.random(n) < 0.8
    st["persistence_time"][:] = 0.001
    st["bias"][:] = 1.0
    st["restrict_2d"][:] = 1 if two_d else 0
    st["vec"][:] = rng.normal(0, 1, 3 * n)
    st["chemotaxis_index"][:] = rng.integers(0, S, n)
    st["chemotaxis_direction"][:] = np.where(rng.random(n) < 0.5, 1, -1)
    if multi:
        st["sensitivity"][:] = rng.uniform(-1, 1, n * S)
    return grid, geo, dens, soa, st, n, mc


def gen_motility():
    rng = np.random.default_rng(41)
    for name, two_d, S, multi in (("motility_2d_legacy", True, 1, False), ("motility_3d_multi", False, 2, True)):
        grid, geo, dens, soa0, st, n, mc = motility_case(rng, two_d, S, multi)
        g = po.Grid(*[int(x) for x in grid], *[float(x) for x in geo[:4]], *[float(x) for x in geo[4:]], 0.0)
        soa = soa0.copy()
        st0 = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
        po.ref_motility_update(soa, mc, n, dens, g, st, 0.1)
        arrays = {k: v for k, v in st0.items() if isinstance(v, np.ndarray)}
        np.savez_compressed(os.path.join(OUT, name + ".npz"), grid=grid, geo=geo, density=dens, soa0=soa0, n=n,
                            max_cells=mc, n_sens=st0["n_sens"], soa_out=soa, vec_out=st["vec"],
                            elapsed_out=st["elapsed"], **{"in_" + k: v for k, v in arrays.items()})


def matlab_case(rng, two_d, S, n=40, mc=48, n_types=2):
    """Inputs for writeMatlabSnapshots: a small grid and cells whose 28-field
    SoA columns all carry values."""
    nx, ny, nz = (12, 10, 1) if two_d else (6, 5, 4)
    grid = np.array([nx, ny, nz, S], np.uint32)
    geo = np.array([20.0, 20.0, 20.0, 0.01, -120.0, -100.0, -10.0 if two_d else -40.0], np.float32)
    dens = rng.uniform(0, 40, nx * ny * nz * S).astype(np.float32)
    soa = np.zeros(28 * mc, np.float32)
    for f in range(23):
        soa[f * mc:f * mc + n] = rng.normal(0, 50, n)
    for f, hi in ((23, n_types), (24, 6), (25, 2)):
        soa[f * mc:f * mc + n] = rng.integers(0, hi, n).astype(np.uint32).view(np.float32)
    soa[26 * mc:28 * mc] = rng.integers(0, 100, 2 * mc).astype(np.uint32).view(np.float32)
    rates = [rng.uniform(0, 10, n * S) for _ in range(4)]
    return grid, geo, dens, soa, rates, n, mc, n_types


def gen_matlab():
    import tempfile
    rng = np.random.default_rng(51)
    for name, two_d, S in (("matlab_2d", True, 2), ("matlab_3d", False, 1)):
        grid, geo, dens, soa, rates, n, mc, n_types = matlab_case(rng, two_d, S)
        g = po.Grid(*[int(x) for x in grid], *[float(x) for x in geo[:4]], *[float(x) for x in geo[4:]], 0.0)
        with tempfile.TemporaryDirectory() as d:
            po.ref_write_matlab(soa, mc, n, n_types, *rates, dens, g, 3, d)
            cells_mat = np.frombuffer(open(os.path.join(d, "output00000003_cells.mat"), "rb").read(), np.uint8)
            env_mat = np.frombuffer(open(os.path.join(d, "output00000003_microenvironment0.mat"), "rb").read(), np.uint8)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), grid=grid, geo=geo, density=dens, soa=soa, n=n,
                            max_cells=mc, n_types=n_types, sec=rates[0], upt=rates[1], sat=rates[2], ne=rates[3],
                            cells_mat=cells_mat, env_mat=env_mat)


def gen_removal():
    """Dead-cell compaction: the reference's removeCell in phase-3 order on a
    28-field SoA with two substrates; indices with repeats and some past the
    count, as the phenotype loop can produce."""
    rng = np.random.default_rng(31)
    mc, n, S = 96, 80, 2
    soa0 = rng.standard_normal(28 * mc).astype(np.float32)
    soa0[23 * mc:28 * mc] = rng.integers(0, 1 << 20, 5 * mc).astype(np.uint32).view(np.float32)
    rates0 = [rng.uniform(0, 10, mc * S) for _ in range(4)]
    indices = np.concatenate([rng.choice(n, 17, replace=False), [79, 3, 3, 85, 0]]).astype(np.uint32)
    soa, rates = soa0.copy(), [r.copy() for r in rates0]
    n_final = po.ref_cells_remove(soa, mc, n, S, *rates, indices)
    np.savez_compressed(os.path.join(OUT, "removal.npz"), max_cells=mc, n=n, S=S, soa0=soa0, sec0=rates0[0],
                        upt0=rates0[1], sat0=rates0[2], ne0=rates0[3], indices=indices, n_final=n_final, soa=soa,
                        sec=rates[0], upt=rates[1], sat=rates[2], ne=rates[3])


def gen_scenario():
    """The reference's parity scenario parity/scenarios/diffusion_only_2d
    (.json / .xml): a 20 x 20 grid over [-200, 200]^2 um, dx 20, one
    substrate (D 1e5, decay 0.1, Dirichlet 38), uniform 38 initially, no
    cells, dt 0.01 min, 2 min (200 steps), saved every minute.  The fields
    after 100 and 200 steps come from the reference's own sweeps and
    applyDirichletBC (Q1 moves the field although it starts at the target)."""
    nx = ny = 20
    subs_p = [(1e5, 0.1, True, 38.0)]
    g = po.make_grid(nx, ny, 1, 1, dx=20.0, dt=0.01, x_min=-200.0, y_min=-200.0)
    subs = po.make_subs(subs_p)
    d = np.full(nx * ny, 38.0, np.float32)
    saved = []
    for step in range(1, 201):
        po.ref_sweeps(d, g, subs)
        po.ref_dirichlet(d, g, subs)
        if step % 100 == 0:
            saved.append(d.copy())
    np.savez_compressed(os.path.join(OUT, "scenario_diffusion_only_2d.npz"), nx=nx, ny=ny,
                        subs=np.array(subs_p, np.float64), steps=np.array([100, 200]), density=np.stack(saved))


if __name__ == "__main__":
    if not po.ref_available():
        sys.exit("oracle/_ref/libpcg_ref.so not built (make -C oracle REF=<reference checkout>)")
    which = sys.argv[1:] or ["diffusion", "secretion", "mechanics", "motility", "matlab", "removal", "scenario"]
    for w in which:
        globals()["gen_" + w]()
    print("golden vectors written to", OUT)
