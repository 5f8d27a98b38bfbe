"""The configurations the bench does not time, at their full sizes: the
plain 3-D simulation (150^3 voxels, four substrates, 200k cells) through the
single-simulation API against the FP64 oracle, and the batched 2-D set (256
instances, sides 32-256, 100-20k cells) against each instance run alone and
against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = np.float64(np.float32(0.01))
DT_MECH = np.float64(np.float32(0.1))


def rel_err(a, b):
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return float((np.abs(np.asarray(a, np.float64) - b) / np.maximum(np.abs(b), 1e-6 * scale)).max())


def positions_close(got64, ref64, got32):
    """FP64 master positions within 1e-4 um of the oracle's, and the SoA's
    FP32 positions their rounding."""
    err = float(np.abs(np.asarray(got64, np.float64).ravel() - ref64).max())
    assert err <= 1e-4, err
    assert np.array_equal(np.asarray(got32, np.float32), np.asarray(got64, np.float64).ravel().astype(np.float32))
    return True


def oracle_inputs(po, inst):
    g = inst.grid
    og = po.make_grid(g.nx, g.ny, g.nz, g.n_substrates, dx=g.dx, dt=g.dt, x_min=g.x_min, y_min=g.y_min,
                      z_min=g.z_min)
    osubs = po.make_subs([(s.diffusion_coefficient, s.decay_rate, bool(s.dirichlet_enabled), s.target_value)
                          for s in inst.substrates[:g.n_substrates]])
    m = inst.mech
    om = po.Mech(m.dt, m.cell_cell_repulsion, m.cell_cell_adhesion, m.max_interaction_distance,
                 m.mechanics_voxel_size, m.mech_grid_nx, m.mech_grid_ny, m.mech_grid_nz)
    dens = np.repeat(inst.initial_values, g.nx * g.ny * g.nz).astype(np.float32)
    return og, osubs, om, dens


def test_plain_3d_full_size_matches_oracle(ctx, pcg, po):
    """150^3 x 4 substrates, 200k cells: one mechanics period (10 sub-steps of
    sweeps, Dirichlet reset and secretion, then forces and AB2) through the
    single-simulation API; density within 1e-5 of the FP64 oracle, FP64
    master positions within 1e-4 um."""
    from pcg import workloads
    inst = workloads.plain_3d()
    g, n = inst.grid, inst.n_cells
    me = pcg.Microenvironment(ctx, g, inst.substrates)
    me.fill(list(inst.initial_values))
    cells = pcg.Cells(ctx, n, g.n_substrates)
    cells.upload(inst.soa, n, n)
    cells.set_secretion(*inst.rates)
    mech = pcg.CellMechanics(ctx, inst.mech, (g.x_min, g.y_min, g.z_min), n)
    steps, acc = 10, 0.0
    for _ in range(steps):
        me.step(cells, 1)
        acc += DT
        if acc >= DT_MECH - 0.5 * DT:
            mech.computeForces(cells)
            mech.integratePositions(cells, 0.1)
            acc = 0.0
    og, osubs, om, dens = oracle_inputs(po, inst)
    soa = inst.soa.copy()
    pm = po.master_positions(soa, n)
    po.run(og, osubs, om, 0.1, dens, soa, n, n, *inst.rates, None, steps, refresh=bool(inst.flags & 1), pos64=pm)
    assert rel_err(me.densityBuffer(), dens) <= 1e-5
    got = cells.download(n)
    assert positions_close(cells.positions64(), pm, got[:3 * n])


def test_batched_2d_full_set(ctx, pcg, po):
    """All 256 instances in one batch for a mechanics period: every 16th
    instance bit-for-bit what it gets alone, and two of them within the
    oracle's tolerances."""
    from pcg import workloads
    insts = workloads.batched_2d()
    assert len(insts) == 256
    steps = 10
    b = pcg.Batch(ctx, insts)
    b.step(steps)
    ctx.sync()
    picked = list(range(0, 256, 16))
    together = {i: (b.density(i), b.cells(i), b.positions64(i)) for i in picked}
    b.close()
    for i in picked:
        a = pcg.Batch(ctx, [insts[i]])
        a.step(steps)
        ctx.sync()
        d, c = a.density(0), a.cells(0)
        a.close()
        assert np.array_equal(together[i][0].view(np.uint32), d.view(np.uint32)), f"density {i}"
        assert np.array_equal(together[i][1].view(np.uint32), c.view(np.uint32)), f"cells {i}"
    for i in (0, 128):
        inst = insts[i]
        og, osubs, om, dens = oracle_inputs(po, inst)
        n = inst.n_cells
        soa = inst.soa.copy()
        pm = po.master_positions(soa, n)
        po.run(og, osubs, om, 0.1, dens, soa, n, n, *inst.rates, None, steps, refresh=bool(inst.flags & 1),
               pos64=pm)
        assert rel_err(together[i][0], dens) <= 1e-5, f"density {i}"
        assert positions_close(together[i][2], pm, together[i][1][:3 * n]), f"cells {i}"
