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
    po.run(og, po.make_subs([(1e5, 0.1, True, 38.0)]), om, 0.1, rd, rs, n, n, *inst.rates, None, steps)
    assert np.abs(dens - rd).max() / np.abs(rd).max() <= 1e-5
    assert np.abs(block[:3 * n].astype(np.float64) - rs[:3 * n]).max() <= 1e-4
    assert np.array_equal(block[27 * n:28 * n].view(np.uint32), rs[27 * n:28 * n].view(np.uint32))
