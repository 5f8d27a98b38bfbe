"""The oracle pinned against the reference: golden vectors produced by the
reference's own shader and secretion code (tests/golden/gen_golden.py), the
known answers of the reference's test suite (tests/test_secretion.py,
tests/test_diffusion.py, tests/test_diffusion_readback.py), and, when
oracle/_ref was built here, live runs of the reference code."""
import glob
import math
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _diff_case(po, path):
    z = np.load(path)
    nx, ny = int(z["nx"]), int(z["ny"])
    subs_p = [(float(a), float(b), bool(c), float(d)) for a, b, c, d in z["subs"]]
    g = po.make_grid(nx, ny, 1, len(subs_p), dx=20.0, dt=0.01, x_min=-0.5 * nx * 20, y_min=-0.5 * ny * 20)
    return z, g, po.make_subs(subs_p)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "diff_*.npz"))),
                         ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_fp32_mode_bit_exact_to_reference_shaders(po, path):
    """OR_FP32_REF is the reference's FP32 operation sequence: bit-exact."""
    z, g, subs = _diff_case(po, path)
    d = z["density0"].copy()
    for k in range(int(z["steps"])):
        po.sweeps(d, g, subs, po.OR_FP32_REF)
        po.dirichlet(d, g, subs)
        assert np.array_equal(d.view(np.uint32), z["density_steps"][k].view(np.uint32)), f"step {k}"


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "diff_*.npz"))),
                         ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_fp64_close_to_reference_shaders(po, path):
    """The FP64 oracle agrees with the reference's FP32 result to 1e-5 relative."""
    z, g, subs = _diff_case(po, path)
    d = z["density0"].copy()
    for k in range(int(z["steps"])):
        po.sweeps(d, g, subs, po.OR_FP64)
        po.dirichlet(d, g, subs)
        ref = z["density_steps"][k].astype(np.float64)
        scale = max(np.abs(ref).max(), 1e-30)
        err = np.abs(d - ref) / np.maximum(np.abs(ref), 1e-6 * scale)
        assert err.max() <= 1e-5, f"step {k}: {err.max():.3e}"


def test_oracle_reproduces_reference_scenario_diffusion_only_2d(po):
    """The reference's own parity scenario (parity/scenarios/diffusion_only_2d:
    20 x 20 over [-200, 200]^2 um, D 1e5, decay 0.1, Dirichlet 38, uniform 38,
    2 min of 0.01 min steps): the FP32 mode bit for bit after 100 and 200
    steps.  The FP64 oracle is within 1e-4 there: the reference's FP32
    roundings over 200 steps of a field that Q1 drives from 38 to ~4000 add
    up to 2.2e-5 (100 steps) and 4.1e-5 (200 steps) of relative error."""
    z = np.load(os.path.join(GOLDEN, "scenario_diffusion_only_2d.npz"))
    subs_p = [(float(a), float(b), bool(c), float(d)) for a, b, c, d in z["subs"]]
    g = po.make_grid(20, 20, 1, 1, dx=20.0, dt=0.01, x_min=-200.0, y_min=-200.0)
    subs = po.make_subs(subs_p)
    d32 = np.full(400, 38.0, np.float32)
    d64 = d32.copy()
    saved = list(z["steps"])
    for step in range(1, max(saved) + 1):
        po.sweeps(d32, g, subs, po.OR_FP32_REF)
        po.dirichlet(d32, g, subs)
        po.sweeps(d64, g, subs, po.OR_FP64)
        po.dirichlet(d64, g, subs)
        if step in saved:
            ref = z["density"][saved.index(step)]
            assert np.array_equal(d32.view(np.uint32), ref.view(np.uint32)), f"step {step}"
            r = ref.astype(np.float64)
            err = np.abs(d64 - r) / np.maximum(np.abs(r), 1e-6 * np.abs(r).max())
            assert err.max() <= 1e-4, f"step {step}: {err.max():.3e}"


def test_secretion_bit_exact_to_reference(po):
    z = np.load(os.path.join(GOLDEN, "secretion.npz"))
    g = po.make_grid(int(z["nx"]), int(z["ny"]), 1, int(z["S"]), dx=20.0, dt=0.01)
    d = z["density0"].copy()
    po.secretion(d, g, z["voxel"], z["volume"], z["sec"], z["upt"], z["sat"], z["ne"], None, 0.01)
    assert np.array_equal(d.view(np.uint32), z["density1"].view(np.uint32))


def _mech_case(po):
    z = np.load(os.path.join(GOLDEN, "mechanics_2d.npz"))
    m = po.mech_params(-500, 500, -500, 500, -10, 10, True, 0.1)
    assert [m.mech_grid_nx, m.mech_grid_ny, m.mech_grid_nz] == list(z["mech"])
    return z, m, int(z["max_cells"]), int(z["n"]), (-500.0, -500.0, -10.0)


def test_mechanics_bins_and_hash_match_reference(po):
    """Bins bit-exact; the reference hash filled in thread order lists each
    voxel's cells exactly as the oracle's stable order."""
    z, m, mc, n, origin = _mech_case(po)
    s = z["soa0"].copy()
    key = po.mech_bin(s, mc, n, m, origin)
    order, start = po.mech_sort(key, m)
    assert np.array_equal(s[27 * mc:27 * mc + n].view(np.uint32), z["soa_forces"][27 * mc:27 * mc + n].view(np.uint32))
    counts = z["hash_counts"]
    assert counts.max() <= 64
    assert np.array_equal(np.diff(start), counts)
    cells = z["hash_cells"]
    for v in np.nonzero(counts)[0]:
        assert np.array_equal(cells[v * 64:v * 64 + counts[v]], order[start[v]:start[v + 1]])


def test_mechanics_forces_match_reference(po):
    z, m, mc, n, origin = _mech_case(po)
    s = z["soa0"].copy()
    key = po.mech_bin(s, mc, n, m, origin)
    order, start = po.mech_sort(key, m)
    cnt, hsh, scale = po.mech_forces(s, mc, n, m, key, order, start)
    ref = z["soa_forces"]
    for f in (3, 4, 5):
        d = np.abs(s[f * mc:f * mc + n].astype(np.float64) - ref[f * mc:f * mc + n])
        assert np.all(d <= 1e-5 * scale + 1e-6), f"field {f}: {d.max():.3e}"
    p, pr = s[22 * mc:22 * mc + n].astype(np.float64), ref[22 * mc:22 * mc + n].astype(np.float64)
    assert np.all(np.abs(p - pr) <= 1e-5 * np.maximum(np.abs(pr), 1.0))
    assert cnt.sum() > n   # the disc is crowded: many contacts


def test_mechanics_integrate_matches_reference(po):
    z, m, mc, n, origin = _mech_case(po)
    s = z["soa_forces"].copy()           # reference forces as velocity input
    po.mech_integrate(s, mc, n, m, origin, 0.1)
    ref = z["soa_integrated"]
    for f in (0, 1, 2):
        assert np.abs(s[f * mc:f * mc + n] - ref[f * mc:f * mc + n]).max() <= 1e-4
    for f in (6, 7, 8):
        assert np.array_equal(s[f * mc:f * mc + n], ref[f * mc:f * mc + n])


# ---- known answers from the reference's own tests ----------------------

def test_secretion_kat_volume_scaled(po):
    """tests/test_secretion.py:66-95: ic = 0.0031175 and rho' = (rho + ic S rho*)
    / (1 + ic (S + U)).  The docstring there quotes ~10.3883, but its own
    numbers give 10.59233 / 1.018705 = 10.39783, which is what its assertion
    (result == formula) checks; this test pins the formula value."""
    g = po.make_grid(1, 1, 1, 1, dx=20.0, dt=0.01)
    d = np.array([10.0], np.float32)
    po.secretion(d, g, np.array([0], np.uint32), np.array([2494.0], np.float32), np.array([5.0]),
                 np.array([1.0]), np.array([38.0]), np.array([0.0]), None, 0.01)
    ic = 0.01 * 2494.0 / 8000.0
    assert abs(ic - 0.0031175) < 1e-12
    expected = (10.0 + ic * 5.0 * 38.0) / (1.0 + ic * 6.0)
    assert abs(float(d[0]) - expected) < 1e-5 and abs(float(d[0]) - 10.39783) < 1e-4


def test_secretion_kat_saturation_and_export(po):
    """tests/test_secretion.py:119-159: fixed point at saturation; net export additive."""
    g = po.make_grid(1, 1, 1, 1, dx=20.0, dt=0.01)
    d = np.array([38.0], np.float32)
    po.secretion(d, g, np.array([0], np.uint32), np.array([2494.0], np.float32), np.array([10.0]),
                 np.array([0.0]), np.array([38.0]), np.array([0.0]), None, 0.01)
    assert float(d[0]) == 38.0
    d = np.array([5.0], np.float32)
    po.secretion(d, g, np.array([0], np.uint32), np.array([2494.0], np.float32), np.array([0.0]),
                 np.array([0.0]), np.array([38.0]), np.array([100.0]), None, 0.01)
    assert abs(float(d[0]) - (5.0 + 0.01 * 100.0 / 8000.0)) < 1e-6


def test_uptake_monotone_to_zero(po):
    """tests/test_secretion.py:98-116."""
    g = po.make_grid(1, 1, 1, 1, dx=20.0, dt=0.01)
    d = np.array([38.0], np.float32)
    prev = 38.0
    for _ in range(50):
        po.secretion(d, g, np.array([0], np.uint32), np.array([2494.0], np.float32), np.array([0.0]),
                     np.array([10.0]), np.array([0.0]), np.array([0.0]), None, 0.01)
        assert 0.0 <= float(d[0]) <= prev
        prev = float(d[0])
    assert prev < 19.0


def test_pure_decay_lod_2d(po):
    """tests/test_diffusion_readback.py:176-234: D = 0, interior rho0/(1+lam dt/2)^(2N)."""
    g = po.make_grid(16, 16, 1, 1, dx=20.0, dt=0.01)
    subs = po.make_subs([(0.0, 0.1, False, 0.0)])
    d = np.full(256, 38.0, np.float32)
    for _ in range(100):
        po.sweeps(d, g, subs)
    expect = 38.0 / (1 + 0.5 * 0.1 * 0.01) ** 200
    inner = d.reshape(16, 16)[1:-1, 1:-1]
    assert np.abs(inner - expect).max() / expect < 1e-5


def test_pure_decay_lod_3d_rule(po):
    """3-D rule: decay split lambda dt / 3 per sweep -> rho0/(1+lam dt/3)^(3N)."""
    g = po.make_grid(8, 8, 8, 1, dx=20.0, dt=0.01)
    subs = po.make_subs([(0.0, 0.3, False, 0.0)])
    d = np.full(512, 20.0, np.float32)
    for _ in range(50):
        po.sweeps(d, g, subs)
    expect = 20.0 / (1 + 0.3 * 0.01 / 3) ** 150
    inner = d.reshape(8, 8, 8)[1:-1, 1:-1, 1:-1]
    assert np.abs(inner - expect).max() / expect < 1e-5


def test_conservation_no_diffusion_no_decay(po):
    """tests/test_diffusion_readback.py:239-258."""
    g = po.make_grid(16, 16, 1, 1, dx=20.0, dt=0.1)
    subs = po.make_subs([(0.0, 0.0, False, 0.0)])
    d = np.full(256, 38.0, np.float32)
    for _ in range(10):
        po.sweeps(d, g, subs)
    assert np.array_equal(d, np.full(256, 38.0, np.float32))


def test_dirichlet_edges_hold_target(po):
    """tests/test_diffusion_readback.py:263-301 (2-D) and the six-face 3-D rule."""
    g = po.make_grid(16, 16, 1, 1, dx=20.0, dt=0.01)
    subs = po.make_subs([(1e5, 0.0, True, 0.0)])
    d = np.full(256, 38.0, np.float32)
    for _ in range(100):
        po.sweeps(d, g, subs)
        po.dirichlet(d, g, subs)
    a = d.reshape(16, 16)
    assert np.all(a[0] == 0) and np.all(a[-1] == 0) and np.all(a[:, 0] == 0) and np.all(a[:, -1] == 0)
    assert a[1:-1, 1:-1].mean() > 0.1
    g3 = po.make_grid(6, 7, 5, 1, dx=20.0, dt=0.01)
    d3 = np.full(6 * 7 * 5, 3.0, np.float32)
    subs3 = po.make_subs([(1e4, 0.1, True, 9.0)])
    po.sweeps(d3, g3, subs3)
    po.dirichlet(d3, g3, subs3)
    b = d3.reshape(5, 7, 6)
    for face in (b[0], b[-1], b[:, 0], b[:, -1], b[:, :, 0], b[:, :, -1]):
        assert np.all(face == 9.0)


def test_thomas_diagonals(po):
    """tests/test_diffusion.py:178-213: b_int = 1+2c+hd, b_bnd = 1+c+hd; a
    one-interior-node line (n = 3) uses b_int with both folds."""
    c = 1e5 * 0.01 / 400.0
    hd = 0.5 * 0.1 * 0.01
    g = po.make_grid(3, 1, 1, 1, dx=20.0, dy=20.0, dt=0.01)
    subs = po.make_subs([(1e5, 0.1, True, 38.0)])
    d = np.array([1.0, 10.0, 1.0], np.float32)
    po.sweep_axis(d, g, subs, 0)
    assert abs(d[1] - (10.0 + 2 * c * 38.0) / (1 + 2 * c + hd)) < 1e-4 and d[0] == 38.0 and d[2] == 38.0


def test_dirichlet_quirk_uniform_target_not_stationary(po):
    """Dirichlet rows use b_bnd and fold c T: a field equal to T moves."""
    z = np.load(os.path.join(GOLDEN, "diff_uniform_T.npz"))
    assert z["density_steps"][-1].max() > 38.5


@pytest.mark.parametrize("shape", [(40, 30, 1), (17, 9, 11)], ids=["2d", "3d"])
def test_consistent_dirichlet_keeps_uniform_target(po, shape):
    """The library's consistent Dirichlet option (not the reference's rule):
    with no decay a uniform field at the target stays there, where the
    reference's rule moves it; away from the boundary lines both agree on a
    field that only varies inside."""
    nx, ny, nz = shape
    g = po.make_grid(nx, ny, nz, 1, dx=20.0, dt=0.01)
    ref = po.make_subs([(1e5, 0.0, True, 38.0)])
    cons = po.make_subs([(1e5, 0.0, True, 38.0, True)])
    a = np.full(nx * ny * nz, 38.0, np.float32)
    b = a.copy()
    for _ in range(20):
        po.sweeps(a, g, cons)
        po.dirichlet(a, g, cons)
        po.sweeps(b, g, ref)
        po.dirichlet(b, g, ref)
    assert np.abs(a.astype(np.float64) - 38.0).max() <= 1e-4
    assert b.max() > 38.5
    # without Dirichlet lines the option changes nothing
    nd_ref = po.make_subs([(1e5, 0.1, False, 0.0)])
    nd_cons = po.make_subs([(1e5, 0.1, False, 0.0, True)])
    rng = np.random.default_rng(3)
    c = rng.uniform(0, 40, nx * ny * nz).astype(np.float32)
    d = c.copy()
    po.sweeps(c, g, nd_ref)
    po.sweeps(d, g, nd_cons)
    assert np.array_equal(c, d)


def test_gradients_central_and_one_sided(po):
    g = po.make_grid(5, 4, 3, 1, dx=20.0, dt=0.01)
    x = np.arange(5, dtype=np.float32)
    d = np.broadcast_to(x[None, None, :] * 2.0 + 0.0, (3, 4, 5)).astype(np.float32).ravel().copy()
    gx, gy, gz = po.gradients(d, g)
    assert np.allclose(gx, 2.0 / 20.0) and np.allclose(gy, 0.0) and np.allclose(gz, 0.0)


def test_port_matches_oracle(po):
    """The FP32 CPU baseline computes the same step as the oracle."""
    rng = np.random.default_rng(5)
    g = po.make_grid(40, 30, 20, 2, dx=20.0, dt=0.01)
    subs = po.make_subs([(1e5, 0.1, True, 38.0), (2e3, 0.4, False, 0.0)])
    d0 = rng.uniform(0, 40, 2 * 40 * 30 * 20).astype(np.float32)
    a, b = d0.copy(), d0.copy()
    for _ in range(3):
        po.sweeps(a, g, subs)
        po.dirichlet(a, g, subs)
        po.port_sweeps(b, g, subs)
        po.port_dirichlet(b, g, subs)
    assert (np.abs(a - b) / np.maximum(np.abs(a), 1e-3)).max() < 1e-5


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref",
                                                    "libpcg_ref.so")), reason="oracle/_ref not built")
def test_live_reference_random_shapes(po):
    """Fresh random 2-D cases against the reference code itself."""
    rng = np.random.default_rng(99)
    for trial in range(20):
        nx, ny = int(rng.integers(1, 40)), int(rng.integers(1, 40))
        S = int(rng.integers(1, 4))
        subs_p = [(float(np.exp(rng.uniform(0, np.log(1e5)))), float(rng.uniform(0, 1)), bool(rng.integers(0, 2)),
                   float(rng.uniform(0, 40))) for _ in range(S)]
        g = po.make_grid(nx, ny, 1, S, dx=float(rng.uniform(5, 30)), dt=0.01)
        subs = po.make_subs(subs_p)
        d0 = rng.uniform(0, 40, S * nx * ny).astype(np.float32)
        a, b = d0.copy(), d0.copy()
        po.ref_sweeps(a, g, subs)
        po.ref_dirichlet(a, g, subs)
        po.sweeps(b, g, subs, po.OR_FP32_REF)
        po.dirichlet(b, g, subs)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (nx, ny, S)


# ---------------------------------------------------------------- motility

def _motility_fixture(po, path):
    f = np.load(path)
    grid, geo = f["grid"], f["geo"]
    g = po.Grid(*[int(x) for x in grid], *[float(x) for x in geo[:4]], *[float(x) for x in geo[4:]], 0.0)
    n, mc, n_sens = int(f["n"]), int(f["max_cells"]), int(f["n_sens"])
    st = po.motility_state(n, n_sens)
    for k in st:
        if isinstance(st[k], np.ndarray):
            st[k] = f["in_" + k].copy()
    return f, g, n, mc, st


@pytest.mark.parametrize("name", ["motility_2d_legacy", "motility_3d_multi"])
def test_motility_matches_reference_golden(po, name):
    """updateMotility (motility.cpp:179-293) with bias 1 and persistence
    below dt: every motile cell's vector is its normalised chemotaxis
    direction times its speed, independent of the random draws; the oracle
    reproduces the reference's output bit for bit (reference density
    indexing, dead and non-motile cells, the single- and multi-substrate
    rules)."""
    f, g, n, mc, st = _motility_fixture(po, os.path.join(GOLDEN, name + ".npz"))
    soa = f["soa0"].copy()
    po.motility_update(soa, mc, n, f["density"], g, st, 0.1, seed=123, step=9)
    assert np.array_equal(st["vec"], f["vec_out"])
    assert np.array_equal(st["elapsed"], f["elapsed_out"])
    assert np.array_equal(soa, f["soa_out"])


def test_motility_draws_are_counter_based(po):
    """Draw k of (seed, cell, step) is a pure function: repeatable, distinct
    across keys, uniform in [0, 1)."""
    u = [po.uniform(5, c, s, k) for c in range(50) for s in range(4) for k in range(3)]
    assert u == [po.uniform(5, c, s, k) for c in range(50) for s in range(4) for k in range(3)]
    assert len(set(u)) == len(u) and min(u) >= 0.0 and max(u) < 1.0
    big = np.array([po.uniform(9, c, 0, 0) for c in range(4000)])
    assert abs(big.mean() - 0.5) < 0.02 and abs(big.var() - 1 / 12) < 0.01


def test_motility_random_walk_unit_speed_and_persistence(po):
    """bias 0: the vector is a unit direction scaled by the speed; with a
    long persistence most cells keep their vector (no resample)."""
    rng = np.random.default_rng(3)
    n, mc = 400, 400
    g = po.Grid(10, 10, 10, 1, 20.0, 20.0, 20.0, 0.01, 0.0, 0.0, 0.0, 0.0)
    dens = np.zeros(1000, np.float32)
    soa = np.zeros(28 * mc, np.float32)
    soa[16 * mc:17 * mc] = 1.5
    soa[25 * mc:26 * mc] = np.ones(mc, np.uint32).view(np.float32)
    st = po.motility_state(n)
    st["is_motile"][:] = 1
    st["bias"][:] = 0.0
    st["restrict_2d"][:] = 0
    st["persistence_time"][:] = 0.001
    po.motility_update(soa, mc, n, dens, g, st, 0.1, seed=1, step=0)
    v = st["vec"].reshape(3, n)
    assert np.allclose(np.linalg.norm(v, axis=0), 1.5, rtol=1e-12)
    prev = st["vec"].copy()
    st["persistence_time"][:] = 1e6          # resample probability 1e-7
    po.motility_update(soa, mc, n, dens, g, st, 0.1, seed=1, step=1)
    assert np.array_equal(st["vec"], prev)
    assert np.allclose(st["elapsed"], 0.1)


def test_motility_live_reference_when_present(po):
    if not po.ref_available():
        pytest.skip("reference library not built here")
    import importlib.util
    spec = importlib.util.spec_from_file_location("gen_golden", os.path.join(GOLDEN, "gen_golden.py"))
    gg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gg)
    rng = np.random.default_rng(77)
    for two_d, S, multi in ((True, 2, True), (False, 1, False), (False, 3, True)):
        grid, geo, dens, soa0, st, n, mc = gg.motility_case(rng, two_d, S, multi)
        g = po.Grid(*[int(x) for x in grid], *[float(x) for x in geo[:4]], *[float(x) for x in geo[4:]], 0.0)
        a, b = soa0.copy(), soa0.copy()
        sa = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
        po.motility_update(a, mc, n, dens, g, sa, 0.1, seed=0, step=0)
        po.ref_motility_update(b, mc, n, dens, g, st, 0.1)
        assert np.array_equal(a, b) and np.array_equal(sa["vec"], st["vec"])


def test_main_loop_motility_phase(po, pcg):
    """or_run_motile: no motile cell leaves the loop as or_run has it; with
    motile cells, the phase runs once per mechanics step, between forces and
    integrate (main.mm:379-387)."""
    from pcg import workloads
    inst = workloads.plain_2d(seed=5, n_cells=120)
    n = inst.n_cells
    g = inst.grid
    og = po.make_grid(g.nx, g.ny, g.nz, 1, dx=g.dx, dt=g.dt, x_min=g.x_min, y_min=g.y_min, z_min=g.z_min)
    om = po.mech_params(-500, 500, -500, 500, -10, 10, True, 0.1)
    subs = po.make_subs([(1e5, 0.1, True, 38.0)])
    soa = inst.soa.astype(np.float32).copy()
    soa[16 * n:17 * n] = 1.0                    # motility speed
    soa.view(np.uint32)[25 * n:26 * n] = 1      # is_alive
    runs = []
    for motile in (False, None, True):
        d, s = np.full(2500, 38.0, np.float32), soa.copy()
        st = po.motility_state(n)
        st["is_motile"][:] = bool(motile)
        if motile is None:
            po.run(og, subs, om, 0.1, d, s, n, n, *inst.rates, None, 25)
        else:
            _, nxt = po.run(og, subs, om, 0.1, d, s, n, n, *inst.rates, None, 25, motility=st, seed=3)
            assert nxt == 2
        runs.append((d, s, st))
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])
    moved = runs[2][1][:2 * n] - runs[1][1][:2 * n]
    el = runs[2][2]["elapsed"]    # float dt_mechanics; 0 or 0.1 where an update resampled
    assert np.abs(moved).max() > 0 and np.all((np.abs(el - 0.2) < 1e-6) | (np.abs(el - 0.1) < 1e-6) | (el == 0))
    assert np.sum(np.abs(el - 0.2) < 1e-6) > n // 2


# ---------------------------------------------------------------- .mat snapshots

@pytest.mark.parametrize("name", ["matlab_2d", "matlab_3d"])
def test_matlab_golden_layout(po, name, tmp_path):
    """The golden files are MATLAB v4 full double matrices with the
    reference's shapes: cells (71 + 7 T + 8 S) x n, microenvironment
    (4 + S) x voxels with FP32 voxel centres; regenerated byte-identical by
    the reference writer when it is built here."""
    f = np.load(os.path.join(GOLDEN, name + ".npz"))
    S, T, n = int(f["grid"][3]), int(f["n_types"]), int(f["n"])
    nx, ny, nz = (int(x) for x in f["grid"][:3])
    (tmp_path / "c.mat").write_bytes(f["cells_mat"].tobytes())
    (tmp_path / "e.mat").write_bytes(f["env_mat"].tobytes())
    cname, cm = po.read_mat4(str(tmp_path / "c.mat"))
    ename, em = po.read_mat4(str(tmp_path / "e.mat"))
    assert cname == "cells" and cm.shape == (71 + 7 * T + 8 * S, n)
    assert ename == "multiscale_microenvironment" and em.shape == (4 + S, nx * ny * nz)
    geo = f["geo"]
    ix = np.arange(nx * ny * nz) % nx
    xc = (np.float32(geo[4]) + (ix.astype(np.float32) + np.float32(0.5)) * np.float32(geo[0])).astype(np.float64)
    assert np.array_equal(em[0], xc)
    assert np.array_equal(cm[0], np.arange(n, dtype=np.float64))
    if po.ref_available():
        g = po.Grid(nx, ny, nz, S, *[float(x) for x in geo[:4]], *[float(x) for x in geo[4:]], 0.0)
        po.ref_write_matlab(f["soa"], int(f["max_cells"]), n, T, f["sec"], f["upt"], f["sat"], f["ne"], f["density"],
                            g, 3, str(tmp_path))
        assert (tmp_path / "output00000003_cells.mat").read_bytes() == f["cells_mat"].tobytes()
        assert (tmp_path / "output00000003_microenvironment0.mat").read_bytes() == f["env_mat"].tobytes()
