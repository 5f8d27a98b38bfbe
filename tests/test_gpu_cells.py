"""Secretion and mechanics on the GPU against the oracle.

Bit-exact: secretion (the FP64 per-cell update of processSecretion on the
same FP32 density), mechanics voxel bins, the sort permutation, the
cell-start table, per-cell neighbour sets (count + hash of neighbour ids),
and the AB2 update on identical velocities.  Forces: within 1e-5 of the
sum of repulsion/adhesion term magnitudes.  Positions after N mechanics
steps: within 1e-4 um."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

O2 = (1e5, 0.1, True, 38.0)


def rel_err(a, b):
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return float((np.abs(np.asarray(a, np.float64) - b) / np.maximum(np.abs(b), 1e-6 * scale)).max())


def make_cells(rng, n, mc, center, r, two_d, radius=8.41, rep=10.0, adh=0.4, relmax=1.25, grid=None):
    soa = np.zeros(28 * mc, np.float32)
    if two_d:
        rr = r * np.sqrt(rng.random(n))
        th = rng.random(n) * 2 * np.pi
        pos = np.stack([center[0] + rr * np.cos(th), center[1] + rr * np.sin(th), np.zeros(n)], 1)
    else:
        v = rng.normal(size=(n, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        pos = np.asarray(center) + v * (r * rng.random(n) ** (1 / 3))[:, None]
    for a in range(3):
        soa[a * mc:a * mc + n] = pos[:, a]
    soa[9 * mc:9 * mc + n] = radius if np.isscalar(radius) else radius[:n]
    soa[11 * mc:11 * mc + n] = 2494.0
    soa[13 * mc:13 * mc + n] = rep
    soa[14 * mc:14 * mc + n] = adh
    soa[15 * mc:15 * mc + n] = relmax
    return soa


def setup_mech(pcg, po, two_d, n, seed, dense=False):
    rng = np.random.default_rng(seed)
    if two_d:
        dom = (-500.0, 500.0, -500.0, 500.0, -10.0, 10.0)
        soa = make_cells(rng, n, n, (0.0, 0.0), 60.0 if dense else 200.0, True)
    else:
        dom = (0.0, 600.0, 0.0, 600.0, 0.0, 600.0)
        soa = make_cells(rng, n, n, (300.0, 300.0, 300.0), 80.0 if dense else 200.0, False,
                         radius=np.clip(rng.normal(8.4, 0.5, n), 5, 12).astype(np.float32))
    mp = pcg.mech_params_for_domain(*dom, two_d, 0.1)
    om = po.mech_params(*dom, two_d, 0.1)
    origin = (dom[0], dom[2], dom[4])
    soa[6 * n:9 * n] = rng.normal(0, 1, 3 * n).astype(np.float32)   # previous velocities
    return soa, mp, om, origin


@pytest.mark.parametrize("two_d,n,dense", [(True, 500, False), (False, 4000, False), (True, 3000, True),
                                           (False, 3000, True)], ids=["2d_cfg0", "3d", "2d_dense", "3d_dense"])
def test_bins_sort_start_and_neighbours_exact(ctx, pcg, po, two_d, n, dense):
    soa, mp, om, origin = setup_mech(pcg, po, two_d, n, 10 + n, dense)
    cells = pcg.Cells(ctx, n, 1)
    cells.upload(soa, n, n)
    mech = pcg.CellMechanics(ctx, mp, origin, n)
    mech.set_diagnostics(True)
    mech.computeForces(cells)
    got = cells.download(n)
    start, order = mech.syncHashPointers(n)
    cnt, hsh = mech.neighbor_stats(n)
    ref = soa.copy()
    key = po.mech_bin(ref, n, n, om, origin)
    oorder, ostart = po.mech_sort(key, om)
    ocnt, ohsh, scale = po.mech_forces(ref, n, n, om, key, oorder, ostart)
    assert np.array_equal(got[27 * n:28 * n].view(np.uint32), key)                  # bins
    assert np.array_equal(start, ostart)                                            # cell-start table
    assert np.array_equal(order, oorder)                                            # permutation
    assert np.array_equal(cnt, ocnt) and np.array_equal(hsh, ohsh)                  # neighbour sets
    if dense:
        assert np.diff(ostart).max() > 64 or not two_d    # past the reference's 64-slot cap
    for f in (3, 4, 5):
        d = np.abs(got[f * n:(f + 1) * n].astype(np.float64) - ref[f * n:(f + 1) * n])
        assert np.all(d <= 1e-5 * scale + 1e-6), f"field {f} max {d.max():.3e}"
    p, pr = got[22 * n:23 * n].astype(np.float64), ref[22 * n:23 * n].astype(np.float64)
    assert np.all(np.abs(p - pr) <= 1e-5 * np.maximum(np.abs(pr), 1.0))


@pytest.mark.parametrize("n", [200_000, 1_500_000], ids=["200k", "1.5M"])
def test_sort_and_start_many_tiles(ctx, pcg, po, n):
    """The stable radix sort over hundreds of 2048-key tiles per pass (a 3 mm
    domain: 100^3 mechanics voxels, 20-bit keys, three passes): bins,
    cell-start table and permutation bit-exact against the oracle."""
    rng = np.random.default_rng(77 + n % 1000)
    dom = (0.0, 3000.0, 0.0, 3000.0, 0.0, 3000.0)
    soa = make_cells(rng, n, n, (1500.0, 1500.0, 1500.0), 1400.0, False)
    mp = pcg.mech_params_for_domain(*dom, False, 0.1)
    om = po.mech_params(*dom, False, 0.1)
    origin = (dom[0], dom[2], dom[4])
    assert po.mech_nvox(om) >= 1 << 17   # more than two 8-bit digits of key
    cells = pcg.Cells(ctx, n, 1)
    cells.upload(soa, n, n)
    mech = pcg.CellMechanics(ctx, mp, origin, n)
    mech.computeForces(cells)
    got = cells.download(n)
    start, order = mech.syncHashPointers(n)
    key = po.mech_bin(soa.copy(), n, n, om, origin)
    oorder, ostart = po.mech_sort(key, om)
    assert np.array_equal(got[27 * n:28 * n].view(np.uint32), key)
    assert np.array_equal(start, ostart)
    assert np.array_equal(order, oorder)


def test_integrate_bit_exact_on_same_velocity(ctx, pcg, po):
    n = 2000
    soa, mp, om, origin = setup_mech(pcg, po, False, n, 3)
    rng = np.random.default_rng(4)
    soa[3 * n:6 * n] = rng.normal(0, 20, 3 * n).astype(np.float32)
    soa[0:n] = np.where(rng.random(n) < 0.05, 599.5, soa[0:n])                    # some clamp
    cells = pcg.Cells(ctx, n, 1)
    cells.upload(soa, n, n)
    mech = pcg.CellMechanics(ctx, mp, origin, n)
    mech.integratePositions(cells, 0.1)
    got = cells.download(n)
    ref = soa.copy()
    po.mech_integrate(ref, n, n, om, origin, 0.1)
    assert np.array_equal(got[:9 * n].view(np.uint32), ref[:9 * n].view(np.uint32))


@pytest.mark.parametrize("two_d", [True, False], ids=["2d", "3d"])
def test_trajectory_within_1e4_um(ctx, pcg, po, two_d):
    """50 mechanics steps (forces + AB2) from a crowded start."""
    n = 500 if two_d else 1500
    soa, mp, om, origin = setup_mech(pcg, po, two_d, n, 20)
    soa[6 * n:9 * n] = 0.0
    cells = pcg.Cells(ctx, n, 1)
    cells.upload(soa, n, n)
    mech = pcg.CellMechanics(ctx, mp, origin, n)
    ref = soa.copy()
    pm = po.master_positions(ref, n)
    for _ in range(50):
        mech.computeForces(cells)
        mech.integratePositions(cells, 0.1)
        key = po.mech_bin(ref, n, n, om, origin)
        oorder, ostart = po.mech_sort(key, om)
        po.mech_forces(ref, n, n, om, key, oorder, ostart)
        po.mech_integrate(ref, n, n, om, origin, 0.1, pos64=pm)
    got = cells.download(n)
    dev64 = cells.positions64()
    dpos = np.abs(dev64.ravel() - pm).max()
    moved = np.abs(pm - soa[:3 * n]).max()
    assert moved > 1.0          # the cells did move
    assert dpos <= 1e-4, dpos   # FP64 master positions against the oracle's
    # the SoA holds the masters' rounding
    assert np.array_equal(got[:3 * n], dev64.ravel().astype(np.float32))
    assert np.abs(got[:3 * n].astype(np.float64) - ref[:3 * n]).max() <= 1e-4


def test_empty_and_single_cell(ctx, pcg):
    mp = pcg.mech_params_for_domain(-100, 100, -100, 100, -10, 10, True)
    cells = pcg.Cells(ctx, 8, 1)
    mech = pcg.CellMechanics(ctx, mp, (-100.0, -100.0, -10.0), 8)
    mech.computeForces(cells)
    mech.integratePositions(cells, 0.1)
    soa = np.zeros(28, np.float32)
    soa[9] = 8.0
    cells.upload(soa, 1, 1)
    mech.update(cells, 0.1)
    out = cells.download(1)
    assert out[3] == 0 and out[4] == 0 and out[22] == 0


def test_mechanics_deterministic(ctx, pcg, po):
    n = 5000
    soa, mp, om, origin = setup_mech(pcg, po, False, n, 8, dense=True)
    outs = []
    for _ in range(2):
        cells = pcg.Cells(ctx, n, 1)
        cells.upload(soa, n, n)
        mech = pcg.CellMechanics(ctx, mp, origin, n)
        for _ in range(3):
            mech.update(cells, 0.1)
        outs.append(cells.download(n))
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))


# ------------------------------------------------------------------ secretion

def secretion_case(pcg, po, nx, ny, nz, S, n, seed):
    rng = np.random.default_rng(seed)
    subs_p = [O2] + [(1e3, 0.2, False, 0.0)] * (S - 1)
    g = pcg.make_grid(nx, ny, nz, S, dx=20.0, dt=0.01)
    og = po.make_grid(nx, ny, nz, S, dx=20.0, dt=0.01)
    nv = nx * ny * nz
    soa = np.zeros(28 * n, np.float32)
    vox = rng.integers(0, nv + 3, n).astype(np.uint32)     # a few out of range
    vox[: n // 10] = 3                                      # a crowded voxel
    soa[26 * n:27 * n] = vox.view(np.float32)
    soa[11 * n:12 * n] = rng.uniform(1000, 4000, n)
    rates = [rng.uniform(0, 10, n * S), rng.uniform(0, 10, n * S), rng.uniform(0, 40, n * S),
             rng.uniform(-50, 50, n * S)]
    active = (rng.random(n) < 0.9).astype(np.uint8)
    d0 = rng.uniform(0, 40, nv * S).astype(np.float32)
    return g, og, pcg.make_substrates(subs_p), po.make_subs(subs_p), soa, vox, rates, active, d0


# grids of 1 voxel (no digit bits: one pass), 16 voxels (one 4-bit pass), up
# to 22-bit voxel indices (three 8-bit passes of the secretion order), and
# stores of one or several 2048-cell tiles
@pytest.mark.parametrize("shape", [(10, 10, 1, 2, 400), (30, 20, 10, 3, 5000), (50, 50, 1, 1, 500),
                                   (1, 1, 1, 1, 300), (4, 4, 1, 2, 5000), (256, 256, 40, 1, 20000),
                                   (128, 128, 128, 2, 7000)])
def test_secretion_bit_exact(ctx, pcg, po, shape):
    nx, ny, nz, S, n = shape
    g, og, subs, osubs, soa, vox, rates, active, d0 = secretion_case(pcg, po, nx, ny, nz, S, n, sum(shape))
    me = pcg.Microenvironment(ctx, g, subs)
    me.setDensityAll(d0)
    cells = pcg.Cells(ctx, n, S)
    cells.upload(soa, n, n)
    cells.set_secretion(*rates, active=active)
    me.applySecretion(cells, 0.01)
    ref = d0.copy()
    po.secretion(ref, og, vox, soa[11 * n:12 * n], *rates, active, 0.01)
    assert np.array_equal(me.densityBuffer().view(np.uint32), ref.view(np.uint32))


def test_secretion_matches_reference_golden(ctx, pcg):
    import os
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "secretion.npz"))
    nx, ny, S = int(z["nx"]), int(z["ny"]), int(z["S"])
    n = len(z["voxel"])
    g = pcg.make_grid(nx, ny, 1, S, dx=20.0, dt=0.01)
    me = pcg.Microenvironment(ctx, g, pcg.make_substrates([O2] * S))
    me.setDensityAll(z["density0"])
    soa = np.zeros(28 * n, np.float32)
    soa[26 * n:27 * n] = z["voxel"].view(np.float32)
    soa[11 * n:12 * n] = z["volume"]
    cells = pcg.Cells(ctx, n, S)
    cells.upload(soa, n, n)
    cells.set_secretion(z["sec"], z["upt"], z["sat"], z["ne"])
    me.applySecretion(cells, 0.01)
    assert np.array_equal(me.densityBuffer().view(np.uint32), z["density1"].view(np.uint32))


def test_remove_matches_reference_fixture(ctx, pcg, po):
    """Dead-cell compaction on the device against the reference's own
    removeCell run in phase-3 order (fixture), the active flags against the
    oracle."""
    import os
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "removal.npz"))
    mc, n, S = int(d["max_cells"]), int(d["n"]), int(d["S"])
    act0 = (np.arange(mc) % 3 != 0).astype(np.uint8)
    cells = pcg.Cells(ctx, mc, S)
    cells.upload(d["soa0"], n, mc)
    cells.set_secretion(*[d[k + "0"][:n * S] for k in ("sec", "upt", "sat", "ne")], active=act0[:n])
    nf = cells.remove(d["indices"])
    assert nf == int(d["n_final"])
    got = cells.download(mc).reshape(28, mc)[:, :nf]
    assert np.array_equal(got.view(np.uint32), d["soa"].reshape(28, mc)[:, :nf].view(np.uint32))
    rates = cells.download_secretion()
    for got_r, k in zip(rates[:4], ("sec", "upt", "sat", "ne")):
        assert np.array_equal(got_r, d[k][:nf * S])
    want_act = act0.copy()
    po.cells_remove(d["soa0"].copy(), mc, n, S, None, None, None, None, want_act, d["indices"])
    assert np.array_equal(rates[4], want_act[:nf])


def test_append_and_remove_then_secretion(ctx, pcg, po):
    """Division and death without re-uploads: cells appended after the
    current ones, secretion, dead cells compacted out (repeats and indices
    past the count included), secretion again; every state bit-exact to the
    oracle, so the secretion order and constants follow the changed
    population."""
    nx, ny, nz, S, n_all, n0 = 30, 20, 10, 3, 5000, 4000
    g, og, subs, osubs, soa, vox, rates, active, d0 = secretion_case(pcg, po, nx, ny, nz, S, n_all, 99)
    me = pcg.Microenvironment(ctx, g, subs)
    me.setDensityAll(d0)
    cells = pcg.Cells(ctx, n_all, S)
    cells.upload(soa, n0, n_all)
    cells.set_secretion(*[r[:n0 * S] for r in rates], active=active[:n0])
    tail = np.ascontiguousarray(soa.reshape(28, n_all)[:, n0:])
    assert cells.append(tail, n_all - n0, n_all - n0, *[r[n0 * S:] for r in rates], active=active[n0:]) == n_all
    me.applySecretion(cells, 0.01)
    ref = d0.copy()
    po.secretion(ref, og, vox, soa[11 * n_all:12 * n_all], *rates, active, 0.01)
    assert np.array_equal(me.densityBuffer().view(np.uint32), ref.view(np.uint32))

    rng = np.random.default_rng(7)
    idx = rng.integers(0, n_all + 50, 700).astype(np.uint32)
    h_soa, h_rates, h_act = soa.copy(), [r.copy() for r in rates], active.copy()
    nf = po.cells_remove(h_soa, n_all, n_all, S, *h_rates, h_act, idx)
    assert cells.remove(idx) == nf
    got = cells.download(n_all).reshape(28, n_all)[:, :nf]
    assert np.array_equal(got.view(np.uint32), h_soa.reshape(28, n_all)[:, :nf].view(np.uint32))
    back = cells.download_secretion()
    for got_r, want in zip(back[:4], h_rates):
        assert np.array_equal(got_r, want[:nf * S])
    assert np.array_equal(back[4], h_act[:nf])

    me.applySecretion(cells, 0.01)
    h_vox = h_soa[26 * n_all:26 * n_all + nf].view(np.uint32)
    po.secretion(ref, og, h_vox, h_soa[11 * n_all:11 * n_all + nf], *[r[:nf * S] for r in h_rates], h_act[:nf],
                 0.01)
    assert np.array_equal(me.densityBuffer().view(np.uint32), ref.view(np.uint32))


def test_remove_then_mechanics_exact(ctx, pcg, po):
    """Bins, cell-start table, permutation and neighbour sets after a
    compaction, against the oracle on the compacted population."""
    n = 3000
    soa, mp, om, origin = setup_mech(pcg, po, False, n, 123, dense=True)
    cells = pcg.Cells(ctx, n, 1)
    cells.upload(soa, n, n)
    idx = np.random.default_rng(8).choice(n, 400, replace=False).astype(np.uint32)
    h = soa.copy()
    nf = po.cells_remove(h, n, n, 0, None, None, None, None, None, idx)
    assert cells.remove(idx) == nf
    mech = pcg.CellMechanics(ctx, mp, origin, n)
    mech.set_diagnostics(True)
    mech.computeForces(cells)
    got = cells.download(n)
    start, order = mech.syncHashPointers(nf)
    cnt, hsh = mech.neighbor_stats(nf)
    key = po.mech_bin(h, n, nf, om, origin)
    oorder, ostart = po.mech_sort(key, om)
    ocnt, ohsh, _ = po.mech_forces(h, n, nf, om, key, oorder, ostart)
    assert np.array_equal(got[27 * n:27 * n + nf].view(np.uint32), key)
    assert np.array_equal(start, ostart)
    assert np.array_equal(order, oorder)
    assert np.array_equal(cnt, ocnt) and np.array_equal(hsh, ohsh)


def test_main_loop_steps_match_oracle(ctx, pcg, po):
    """Sweeps -> Dirichlet -> secretion -> mechanics every 10th sub-step
    (src/main.mm:341-391) through the plain API, against or_run."""
    from pcg import workloads
    inst = workloads.plain_2d()
    g, n = inst.grid, inst.n_cells
    og = po.make_grid(g.nx, g.ny, g.nz, g.n_substrates, dx=g.dx, dt=g.dt, x_min=g.x_min, y_min=g.y_min,
                      z_min=g.z_min)
    osubs = po.make_subs([(1e5, 0.1, True, 38.0)])
    om = po.mech_params(-500, 500, -500, 500, -10, 10, True, 0.1)
    me = pcg.Microenvironment(ctx, g, inst.substrates)
    me.fill([38.0])
    cells = pcg.Cells(ctx, n, 1)
    cells.upload(inst.soa, n, n)
    cells.set_secretion(*inst.rates)
    mech = pcg.CellMechanics(ctx, inst.mech, (g.x_min, g.y_min, -10.0), n)
    acc = 0.0
    steps = 60
    for _ in range(steps):
        me.step(cells, 1)
        acc += np.float64(np.float32(0.01))
        if acc >= np.float64(np.float32(0.1)) - 0.5 * np.float64(np.float32(0.01)):
            mech.computeForces(cells)
            mech.integratePositions(cells, 0.1)
            acc = 0.0
    dens = np.full(2500, 38.0, np.float32)
    soa = inst.soa.copy()
    pm = po.master_positions(soa, n)
    po.run(og, osubs, om, 0.1, dens, soa, n, n, *inst.rates, None, steps, pos64=pm)
    assert rel_err(me.densityBuffer(), dens) <= 1e-5
    got = cells.download(n)
    assert np.abs(cells.positions64().ravel() - pm).max() <= 1e-4
    assert np.abs(got[:3 * n].astype(np.float64) - soa[:3 * n]).max() <= 1e-4


def test_main_loop_with_voxel_refresh_matches_oracle(ctx, pcg, po):
    """The single-simulation API with voxel indices refreshed after every
    integrate (pcg_cells_set_voxel_refresh) against or_run with the same
    rule: density, master positions and voxel indices."""
    from pcg import workloads
    inst = workloads.plain_2d(n_cells=800)
    g, n = inst.grid, inst.n_cells
    me = pcg.Microenvironment(ctx, g, inst.substrates)
    me.fill([38.0])
    cells = pcg.Cells(ctx, n, 1)
    cells.upload(inst.soa, n, n)
    cells.set_secretion(*inst.rates)
    cells.set_voxel_refresh(me)
    mech = pcg.CellMechanics(ctx, inst.mech, (g.x_min, g.y_min, -10.0), n)
    acc = 0.0
    steps = 60
    for _ in range(steps):
        me.step(cells, 1)
        acc += np.float64(np.float32(0.01))
        if acc >= np.float64(np.float32(0.1)) - 0.5 * np.float64(np.float32(0.01)):
            mech.computeForces(cells)
            mech.integratePositions(cells, 0.1)
            acc = 0.0
    og = po.make_grid(g.nx, g.ny, g.nz, 1, dx=g.dx, dt=g.dt, x_min=g.x_min, y_min=g.y_min, z_min=g.z_min)
    om = po.mech_params(-500, 500, -500, 500, -10, 10, True, 0.1)
    dens = np.full(2500, 38.0, np.float32)
    soa = inst.soa.copy()
    pm = po.master_positions(soa, n)
    po.run(og, po.make_subs([(1e5, 0.1, True, 38.0)]), om, 0.1, dens, soa, n, n, *inst.rates, None, steps,
           refresh=True, pos64=pm)
    got = cells.download(n)
    assert rel_err(me.densityBuffer(), dens) <= 1e-5
    assert np.abs(cells.positions64().ravel() - pm).max() <= 1e-4
    moved = np.sum(got[26 * n:27 * n].view(np.uint32) != inst.soa[26 * n:27 * n].view(np.uint32))
    assert moved > 0                                    # some cells changed voxel
    assert np.array_equal(got[26 * n:27 * n].view(np.uint32), soa[26 * n:27 * n].view(np.uint32))
    cells.set_voxel_refresh(None, False)


def test_remove_and_append_edge_cases(ctx, pcg):
    """Removing nothing, removing every cell, appending to an empty store,
    and an append past max_cells refused without changing the store."""
    n, S = 50, 2
    soa = np.arange(28 * n, dtype=np.float32)
    cells = pcg.Cells(ctx, n, S)
    cells.upload(soa, n, n)
    assert cells.remove([]) == n
    assert np.array_equal(cells.download(n).view(np.uint32), soa.view(np.uint32))
    assert cells.remove(np.arange(n + 5)) == 0
    assert cells.append(soa, 10, n) == 10
    got = cells.download(n).reshape(28, n)[:, :10]
    assert np.array_equal(got.view(np.uint32), soa.reshape(28, n)[:, :10].view(np.uint32))
    rates = cells.download_secretion()
    assert all(np.all(r == 0.0) for r in rates[:4]) and np.all(rates[4] == 1)
    with pytest.raises(pcg.PcgError):
        cells.append(soa, 41, n)
    assert cells.count() == 10
