"""The C++ drop-ins (host/pcg_host.h) driven by the main-loop twin
(host/sim_main.cpp, built as pcg_sim) against the oracle's main loop."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SIM = os.path.join(ROOT, "physicell-mac-metal_b200", "pcg_sim")


def test_main_loop_twin_matches_oracle(tmp_path, pcg, po):
    from pcg import workloads
    inst = workloads.plain_2d(seed=77)
    n = inst.n_cells
    path = tmp_path / "cells.bin"
    with open(path, "wb") as f:
        np.array([n, n], np.uint32).tofile(f)
        inst.soa.astype(np.float32).tofile(f)
        for r in inst.rates:
            np.asarray(r, np.float64).tofile(f)
    out = tmp_path / "out.bin"
    steps = 45
    res = subprocess.run([SIM, str(path), str(steps), str(out)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    assert "Diffusion (GPU)" in res.stdout
    raw = np.fromfile(out, np.float32)
    dens, block = raw[:2500], raw[2500:]
    g = inst.grid
    og = po.make_grid(g.nx, g.ny, g.nz, 1, dx=g.dx, dt=g.dt, x_min=g.x_min, y_min=g.y_min, z_min=g.z_min)
    om = po.mech_params(-500, 500, -500, 500, -10, 10, True, 0.1)
    rd = np.full(2500, 38.0, np.float32)
    rs = inst.soa.copy()
    po.run(og, po.make_subs([(1e5, 0.1, True, 38.0)]), om, 0.1, rd, rs, n, n, *inst.rates, None, steps,
           pos64=po.master_positions(rs, n))
    assert np.abs(dens - rd).max() / np.abs(rd).max() <= 1e-5
    assert np.abs(block[:3 * n].astype(np.float64) - rs[:3 * n]).max() <= 1e-4
    assert np.array_equal(block[27 * n:28 * n].view(np.uint32), rs[27 * n:28 * n].view(np.uint32))


def _write_motility(path, st, n):
    with open(path, "wb") as f:
        for k in ("persistence_time", "elapsed", "bias"):
            np.asarray(st[k], np.float64).tofile(f)
        np.asarray(st["vec"], np.float64).tofile(f)          # x[n], y[n], z[n]
        for k, t in (("is_motile", np.uint32), ("restrict_2d", np.uint32),
                     ("chemotaxis_index", np.int32), ("chemotaxis_direction", np.int32)):
            np.asarray(st[k], t).tofile(f)
        ns = st["n_sens"] if st["sensitivity"] is not None else 0
        np.array([ns], np.uint32).tofile(f)
        if ns:
            np.asarray(st["sensitivity"], np.float64).tofile(f)


@pytest.mark.parametrize("n_sens", [0, 1])
def test_main_loop_twin_with_motility_and_mat_frames(tmp_path, pcg, po, n_sens):
    """main.mm:379-387 with updateMotility between forces and integrate, and
    the .mat frames of main.mm:299 / :424, through MotilityData,
    updateMotility, SnapshotWriter and writeMatlabSnapshots of pcg_host.h."""
    from pcg import workloads
    inst = workloads.plain_2d(seed=78)
    n = inst.n_cells
    rng = np.random.default_rng(11 + n_sens)
    soa = inst.soa.astype(np.float32).copy()
    soa[16 * n:17 * n] = rng.uniform(0.2, 2.0, n)               # motility speed
    soa.view(np.uint32)[25 * n:26 * n] = rng.random(n) < 0.9    # is_alive
    st = po.motility_state(n, n_sens)
    st["is_motile"][:] = rng.random(n) < 0.8
    st["persistence_time"][:] = rng.uniform(0.05, 5.0, n)       # several direction changes in the run
    st["bias"][:] = rng.uniform(0.0, 1.0, n)
    st["chemotaxis_direction"][:] = rng.choice([-1, 1], n)
    if n_sens:
        st["sensitivity"][:] = rng.uniform(-1.0, 1.0, n) * (rng.random(n) < 0.6)
    cells_bin, mot_bin = tmp_path / "cells.bin", tmp_path / "mot.bin"
    with open(cells_bin, "wb") as f:
        np.array([n, n], np.uint32).tofile(f)
        soa.tofile(f)
        for r in inst.rates:
            np.asarray(r, np.float64).tofile(f)
    _write_motility(mot_bin, st, n)
    out, mat = tmp_path / "out.bin", tmp_path / "mat"
    mat.mkdir()
    steps, seed = 45, 4242
    res = subprocess.run([SIM, str(cells_bin), str(steps), str(out), "--motility", str(mot_bin),
                          "--seed", str(seed), "--mat", str(mat)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    raw = np.fromfile(out, np.uint8)
    nb = 4 * (2500 + 28 * n)
    dens = raw[:4 * 2500].view(np.float32)
    block = raw[4 * 2500:nb].view(np.float32)
    mot = raw[nb:].view(np.float64)
    elapsed, vec = mot[:n], mot[n:4 * n]

    g = inst.grid
    og = po.make_grid(g.nx, g.ny, g.nz, 1, dx=g.dx, dt=g.dt, x_min=g.x_min, y_min=g.y_min, z_min=g.z_min)
    om = po.mech_params(-500, 500, -500, 500, -10, 10, True, 0.1)
    rd = np.full(2500, 38.0, np.float32)
    rs = soa.copy()
    _, next_step = po.run(og, po.make_subs([(1e5, 0.1, True, 38.0)]), om, 0.1, rd, rs, n, n, *inst.rates, None,
                          steps, motility=st, seed=seed, mot_step=0, layout=po.MOT_REF,
                          pos64=po.master_positions(rs, n))
    assert next_step == 4                                       # mechanics every 10 diffusion steps
    assert np.abs(dens - rd).max() / np.abs(rd).max() <= 1e-5
    assert np.abs(block[:3 * n].astype(np.float64) - rs[:3 * n]).max() <= 1e-3
    assert np.abs(block[3 * n:6 * n].astype(np.float64) - rs[3 * n:6 * n]).max() <= 1e-3
    assert np.array_equal(elapsed, st["elapsed"])               # same draws decide every resample
    # the chemotaxis direction is a gradient of densities that agree to 1e-5
    # relative, so the vectors (speed <= 2) agree to about that much
    assert np.abs(vec - st["vec"]).max() <= 1e-4
    assert np.abs(vec).max() > 0                                # motility did act

    # frame 0: the state before the loop; frame 1: the state after it
    name, env0 = po.read_mat4(str(mat / "output00000000_microenvironment0.mat"))
    assert name == "multiscale_microenvironment" and env0.shape == (5, 2500)
    assert np.all(env0[4] == 38.0)
    _, c0 = po.read_mat4(str(mat / "output00000000_cells.mat"))
    assert np.array_equal(c0[1:4], soa[:3 * n].reshape(3, n).astype(np.float64))
    _, env1 = po.read_mat4(str(mat / "output00000001_microenvironment0.mat"))
    assert np.array_equal(env1[4], dens.astype(np.float64))
    _, c1 = po.read_mat4(str(mat / "output00000001_cells.mat"))
    assert np.array_equal(c1[0], np.arange(n, dtype=np.float64))
    assert np.array_equal(c1[1:4], block[:3 * n].reshape(3, n).astype(np.float64))
