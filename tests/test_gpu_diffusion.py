"""Diffusion sweeps on the GPU against the FP64 oracle (1e-5 relative per
field, the stated tolerance) and against the reference's golden vectors."""
import glob
import os
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-5   # max over voxels |gpu - oracle| / max(|oracle|, 1e-6 max|oracle|)


def rel_err(a, b):
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return float((np.abs(np.asarray(a, np.float64) - b) / np.maximum(np.abs(b), 1e-6 * scale)).max())


def both_grids(pcg, po, nx, ny, nz, subs_p, dx=20.0, dt=0.01):
    S = len(subs_p)
    g = pcg.make_grid(nx, ny, nz, S, dx=dx, dt=dt, x_min=-nx * dx / 2, y_min=-ny * dx / 2, z_min=0.0)
    og = po.make_grid(nx, ny, nz, S, dx=dx, dt=dt, x_min=-nx * dx / 2, y_min=-ny * dx / 2, z_min=0.0)
    return g, pcg.make_substrates(subs_p), og, po.make_subs(subs_p)


O2 = (1e5, 0.1, True, 38.0)
CASES = [
    ("cfg0_50x50", 50, 50, 1, [O2]),
    ("2d_two_subs", 37, 21, 1, [O2, (2e3, 0.5, False, 0.0)]),
    ("3d_small", 24, 17, 11, [O2, (5e3, 0.3, True, 4.0)]),
    ("3d_cube_40", 40, 40, 40, [O2]),
    ("3d_odd", 33, 35, 31, [(3e4, 0.7, False, 0.0), O2, (1e3, 0.05, True, 12.0)]),
    ("n3_lines", 3, 3, 3, [O2]),
    ("n4_lines", 4, 5, 4, [O2, (1e4, 0.2, False, 0.0)]),
    ("n2_lines", 2, 9, 2, [O2]),
    ("n1_lines", 1, 7, 1, [O2]),
    ("thin_x", 1, 1, 9, [O2]),
    ("long_x_global", 800, 3, 1, [O2]),
    ("long_y_global", 5, 600, 1, [O2]),
    ("long_z_global", 6, 4, 530, [(1e4, 0.1, True, 3.0)]),
    ("wide_y", 70, 3, 1, [(1e5, 0.0, True, 0.0)]),
    ("x_bulk_300", 300, 7, 1, [O2]),                     # x lines past a tensor box: one bulk copy per tile
    ("y_bulk_400", 9, 400, 1, [O2, (2e3, 0.2, False, 0.0)]),   # column tiles by per-row bulk copies
    ("z_bulk_270", 5, 6, 270, [(1e4, 0.1, True, 3.0)]),
    ("3d_w16_groups", 44, 13, 9, [O2, (4e3, 0.3, True, 2.0)]),  # 12-column remainder: 16-wide, 2-slab tiles
    ("3d_x70", 70, 9, 12, [O2, (4e3, 0.3, True, 2.0)]),         # z: 32-wide tiles + a 6-column remainder
    ("3d_x130", 130, 6, 8, [(2e4, 0.1, True, 5.0)]),            # x rows past 128, z remainder of 2 columns
    ("3d_plane_150", 150, 150, 5, [O2]),                          # x-y planes of ~93 KB: 2 CTAs per SM
    ("3d_rows_200", 40, 200, 3, [O2, (3e3, 0.2, False, 0.0)]),   # 200 rows: two per plane thread
]


@pytest.mark.parametrize("name,nx,ny,nz,subs_p", CASES, ids=[c[0] for c in CASES])
def test_step_matches_oracle(ctx, pcg, po, name, nx, ny, nz, subs_p):
    g, subs, og, osubs = both_grids(pcg, po, nx, ny, nz, subs_p)
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    d0 = rng.uniform(0.0, 40.0, nx * ny * nz * len(subs_p)).astype(np.float32)
    me = pcg.Microenvironment(ctx, g, subs)
    me.setDensityAll(d0)
    ref = d0.copy()
    for k in range(5):
        me.step(None, 1)
        po.sweeps(ref, og, osubs)
        po.dirichlet(ref, og, osubs)
        got = me.densityBuffer()
        assert rel_err(got, ref) <= TOL, f"step {k}: {rel_err(got, ref):.3e}"


def test_sweeps_only_then_dirichlet_equals_fused_step(ctx, pcg, po):
    """simulateDiffusionDecay + applyDirichletBC (the reference's two calls)
    gives bit-for-bit the fused step."""
    for (nx, ny, nz) in [(50, 50, 1), (30, 20, 10)]:
        g, subs, og, osubs = both_grids(pcg, po, nx, ny, nz, [O2, (3e3, 0.2, True, 1.0)])
        d0 = np.random.default_rng(1).uniform(0, 40, nx * ny * nz * 2).astype(np.float32)
        a = pcg.Microenvironment(ctx, g, subs)
        b = pcg.Microenvironment(ctx, g, subs)
        a.setDensityAll(d0)
        b.setDensityAll(d0)
        for _ in range(3):
            a.simulateDiffusionDecay(1)
            a.applyDirichletBC()
            b.step(None, 1)
        assert np.array_equal(a.densityBuffer().view(np.uint32), b.densityBuffer().view(np.uint32))
        # and the sweeps alone match the oracle's sweeps alone
        c = pcg.Microenvironment(ctx, g, subs)
        c.setDensityAll(d0)
        c.simulateDiffusionDecay(2)
        ref = d0.copy()
        po.sweeps(ref, og, osubs)
        po.sweeps(ref, og, osubs)
        assert rel_err(c.densityBuffer(), ref) <= TOL


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "diff_*.npz"))),
                         ids=lambda p: os.path.basename(p)[:-4])
def test_matches_reference_golden_vectors(ctx, pcg, path):
    z = np.load(path)
    nx, ny = int(z["nx"]), int(z["ny"])
    subs_p = [(float(a), float(b), bool(c), float(d)) for a, b, c, d in z["subs"]]
    g = pcg.make_grid(nx, ny, 1, len(subs_p), dx=20.0, dt=0.01, x_min=-0.5 * nx * 20, y_min=-0.5 * ny * 20)
    me = pcg.Microenvironment(ctx, g, pcg.make_substrates(subs_p))
    me.setDensityAll(z["density0"])
    for k in range(int(z["steps"])):
        me.step(None, 1)
        assert rel_err(me.densityBuffer(), z["density_steps"][k]) <= TOL


def test_long_run_config0_field(ctx, pcg, po):
    """300 steps of the 50x50 O2 field from a random start stay within 1e-5."""
    g, subs, og, osubs = both_grids(pcg, po, 50, 50, 1, [O2])
    d0 = np.random.default_rng(7).uniform(0, 40, 2500).astype(np.float32)
    me = pcg.Microenvironment(ctx, g, subs)
    me.setDensityAll(d0)
    me.step(None, 300)
    ref = d0.copy()
    for _ in range(300):
        po.sweeps(ref, og, osubs)
        po.dirichlet(ref, og, osubs)
    assert rel_err(me.densityBuffer(), ref) <= TOL


def test_pure_decay_known_answer_3d(ctx, pcg):
    g = pcg.make_grid(20, 20, 20, 1, dx=20.0, dt=0.01)
    me = pcg.Microenvironment(ctx, g, pcg.make_substrates([(0.0, 0.3, False, 0.0)]))
    me.fill([20.0])
    me.simulateDiffusionDecay(100)
    expect = 20.0 / (1 + 0.3 * 0.01 / 3) ** 300
    inner = me.densityBuffer().reshape(20, 20, 20)[1:-1, 1:-1, 1:-1]
    assert np.abs(inner - expect).max() / expect < 1e-5


def test_deterministic(ctx, pcg):
    g = pcg.make_grid(60, 50, 40, 2, dx=20.0, dt=0.01)
    subs = pcg.make_substrates([O2, (1e3, 0.2, False, 0.0)])
    d0 = np.random.default_rng(2).uniform(0, 40, 60 * 50 * 40 * 2).astype(np.float32)
    outs = []
    for _ in range(2):
        me = pcg.Microenvironment(ctx, g, subs)
        me.setDensityAll(d0)
        me.step(None, 4)
        outs.append(me.densityBuffer())
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))


def test_gradients_match_oracle(ctx, pcg, po):
    g, subs, og, osubs = both_grids(pcg, po, 19, 13, 7, [O2, (1e3, 0.1, False, 0.0)])
    d0 = np.random.default_rng(4).uniform(0, 40, 19 * 13 * 7 * 2).astype(np.float32)
    me = pcg.Microenvironment(ctx, g, subs)
    me.setDensityAll(d0)
    gx, gy, gz = me.computeGradients()
    ox, oy, oz = po.gradients(d0, og)
    for a, b in ((gx, ox), (gy, oy), (gz, oz)):
        assert np.abs(a - b).max() <= 1e-6 * max(1.0, np.abs(b).max())


def test_size_mismatch_is_an_error(ctx, pcg):
    g = pcg.make_grid(8, 8, 1, 1)
    me = pcg.Microenvironment(ctx, g, pcg.make_substrates([O2]))
    with pytest.raises(pcg.PcgError):
        me.setDensityAll(np.zeros(10, np.float32))


@pytest.mark.parametrize("shape", [(50, 50, 1), (41, 37, 23), (150, 150, 1)], ids=["2d", "3d", "2d_150"])
def test_consistent_dirichlet_matches_oracle(ctx, pcg, po, shape):
    """The consistent Dirichlet option on the device against the oracle's,
    on a field with structure; and a uniform field at the target stays
    there (no decay)."""
    nx, ny, nz = shape
    rng = np.random.default_rng(nx + ny + nz)
    params = [(1e5, 0.1, True, 38.0, True), (3e3, 0.3, True, 5.0, True), (2e4, 0.0, False, 0.0, True)]
    g = pcg.make_grid(nx, ny, nz, 3, dx=20.0, dt=0.01)
    me = pcg.Microenvironment(ctx, g, pcg.make_substrates(params))
    d0 = rng.uniform(0, 40, 3 * nx * ny * nz).astype(np.float32)
    me.setDensityAll(d0)
    me.step(None, 5)
    og = po.make_grid(nx, ny, nz, 3, dx=20.0, dt=0.01)
    osubs = po.make_subs(params)
    ref = d0.copy()
    for _ in range(5):
        po.sweeps(ref, og, osubs)
        po.dirichlet(ref, og, osubs)
    assert rel_err(me.densityBuffer(), ref) <= 1e-5
    flat = [(1e5, 0.0, True, 38.0, True)]
    g1 = pcg.make_grid(nx, ny, nz, 1, dx=20.0, dt=0.01)
    m1 = pcg.Microenvironment(ctx, g1, pcg.make_substrates(flat))
    m1.fill([38.0])
    m1.step(None, 20)
    assert np.abs(m1.densityBuffer().astype(np.float64) - 38.0).max() <= 1e-4
    me.close()
    m1.close()



def test_reference_scenario_diffusion_only_2d(ctx, pcg, po):
    """The reference's parity scenario diffusion_only_2d (20 x 20 over
    [-200, 200]^2 um, D 1e5, decay 0.1, Dirichlet 38, uniform 38 at the start,
    2 min at dt 0.01) after 100 and 200 steps: against the FP64 oracle and
    against the reference's own sweeps and applyDirichletBC run on the CPU
    (golden), within 1e-4 relative.  Over 200 FP32 steps of a field that Q1
    drives from 38 to ~4000 the reference's own FP32 result is 4.1e-5 from
    the FP64 oracle, so the 5-step bar of 1e-5 does not apply here."""
    z = np.load(os.path.join(GOLDEN, "scenario_diffusion_only_2d.npz"))
    subs_p = [(float(a), float(b), bool(c), float(d)) for a, b, c, d in z["subs"]]
    g = pcg.make_grid(20, 20, 1, 1, dx=20.0, dt=0.01, x_min=-200.0, y_min=-200.0)
    og = po.make_grid(20, 20, 1, 1, dx=20.0, dt=0.01, x_min=-200.0, y_min=-200.0)
    osubs = po.make_subs(subs_p)
    me = pcg.Microenvironment(ctx, g, pcg.make_substrates(subs_p))
    me.setDensityAll(np.full(400, 38.0, np.float32))
    ref64 = np.full(400, 38.0, np.float32)
    done = 0
    for k, steps in enumerate(z["steps"]):
        me.step(None, int(steps) - done)
        for _ in range(int(steps) - done):
            po.sweeps(ref64, og, osubs)
            po.dirichlet(ref64, og, osubs)
        done = int(steps)
        got = me.densityBuffer()
        assert rel_err(got, ref64) <= 1e-4, f"{steps} steps vs oracle: {rel_err(got, ref64):.3e}"
        assert rel_err(got, z["density"][k]) <= 1e-4, f"{steps} steps vs reference: {rel_err(got, z['density'][k]):.3e}"
