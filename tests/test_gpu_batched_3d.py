"""The benched configuration at its own size: all 64 batched 3-D instances
(sides 40-120 voxels, two substrates, 1k-100k cells in central spheres;
39.9 M voxels and 3.0 M cells) in one batch, one mechanics period (10
diffusion sub-steps of sweeps, Dirichlet reset and secretion, then one
mechanics step, voxel indices refreshed after it), as the bench times it.

Against the FP64 oracle, for the largest grid, the densest instance, the
instance with the most cells, the smallest grid and the instance whose drug
decays least: density within 1e-5 relative, FP64 master positions within
1e-4 um; the mechanics step's bins, sort permutation, cell-start table and
per-cell neighbour sets bit-exact (reference rules: shaders/diffusion_2d.
metal:28-292 with the 3-D extension, shaders/mechanics.metal:27-216,
shaders/integrate.metal:31-80, src/cell_phenotype.cpp:526-564).  Every 8th
instance also bit for bit what it gets alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 10


def rel_err(a, b):
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return float((np.abs(np.asarray(a, np.float64) - b) / np.maximum(np.abs(b), 1e-6 * scale)).max())


def picks(insts):
    side = np.array([i.grid.nx for i in insts])
    cells = np.array([i.n_cells for i in insts])
    density = cells / side.astype(np.float64) ** 3
    drug_decay = np.array([i.substrates[1].decay_rate for i in insts])
    out = {"largest": int(np.argmax(side)), "densest": int(np.argmax(density)), "most_cells": int(np.argmax(cells)),
           "smallest": int(np.argmin(side)), "slowest_drug_decay": int(np.argmin(drug_decay))}
    return out


@pytest.fixture(scope="module")
def batched(ctx, pcg):
    from pcg import workloads
    insts = workloads.batched_3d()
    assert len(insts) == 64
    b = pcg.Batch(ctx, insts)
    b.set_diagnostics(True)
    b.step(STEPS)
    ctx.sync()
    chosen = sorted(set(picks(insts).values()) | set(range(0, 64, 8)))
    res = {}
    for i in chosen:
        start, order, cnt, hsh = b.mech_bins(i, stats=True)
        res[i] = {"density": b.density(i), "cells": b.cells(i), "pos64": b.positions64(i), "start": start,
                  "order": order, "cnt": cnt, "hash": hsh}
    totals = b.totals()
    b.close()
    return insts, res, totals


def test_workload_is_the_benched_size(batched):
    insts, _, (voxels, voxel_subs, cells) = batched
    assert voxels == sum(i.grid.nx * i.grid.ny * i.grid.nz for i in insts)
    assert voxels > 39_000_000 and cells > 3_000_000 and voxel_subs == 2 * voxels
    p = picks(insts)
    assert insts[p["largest"]].grid.nx >= 115 and insts[p["smallest"]].grid.nx <= 45
    assert insts[p["most_cells"]].n_cells >= 95_000


@pytest.mark.parametrize("which", ["largest", "densest", "most_cells", "smallest", "slowest_drug_decay"])
def test_instance_matches_oracle(batched, po, which):
    insts, res, _ = batched
    i = picks(insts)[which]
    inst, r = insts[i], res[i]
    g, m, n = inst.grid, inst.mech, inst.n_cells
    og = po.make_grid(g.nx, g.ny, g.nz, g.n_substrates, dx=g.dx, dt=g.dt, x_min=g.x_min, y_min=g.y_min,
                      z_min=g.z_min)
    osubs = po.make_subs([(s.diffusion_coefficient, s.decay_rate, bool(s.dirichlet_enabled), s.target_value)
                          for s in inst.substrates[:g.n_substrates]])
    om = po.Mech(m.dt, m.cell_cell_repulsion, m.cell_cell_adhesion, m.max_interaction_distance,
                 m.mechanics_voxel_size, m.mech_grid_nx, m.mech_grid_ny, m.mech_grid_nz)
    origin = (g.x_min, g.y_min, g.z_min)
    # the mechanics step bins the positions the period started from
    # (secretion does not move cells)
    start_soa = inst.soa.copy()
    key = po.mech_bin(start_soa, n, n, om, origin)
    oorder, ostart = po.mech_sort(key, om)
    ocnt, ohsh, _ = po.mech_forces(start_soa, n, n, om, key, oorder, ostart)
    assert np.array_equal(r["cells"][27 * n:28 * n].view(np.uint32), key), "bins"
    assert np.array_equal(r["start"], ostart), "cell-start table"
    assert np.array_equal(r["order"], oorder), "sort permutation"
    assert np.array_equal(r["cnt"], ocnt) and np.array_equal(r["hash"], ohsh), "neighbour sets"
    assert ocnt.sum() > 0
    # the whole period
    dens = np.repeat(inst.initial_values, g.nx * g.ny * g.nz).astype(np.float32)
    soa = inst.soa.copy()
    pm = po.master_positions(soa, n)
    po.run(og, osubs, om, 0.1, dens, soa, n, n, *inst.rates, None, STEPS, refresh=bool(inst.flags & 1), pos64=pm)
    assert rel_err(r["density"], dens) <= 1e-5
    assert float(np.abs(r["pos64"].ravel() - pm).max()) <= 1e-4
    assert np.array_equal(r["cells"][:3 * n], r["pos64"].ravel().astype(np.float32))
    assert float(np.abs(pm - inst.soa[:3 * n]).max()) > 1e-3     # the cells moved


def test_every_eighth_instance_same_alone(batched, ctx, pcg):
    insts, res, _ = batched
    for i in range(0, 64, 8):
        a = pcg.Batch(ctx, [insts[i]])
        a.step(STEPS)
        ctx.sync()
        d, c, p = a.density(0), a.cells(0), a.positions64(0)
        a.close()
        assert np.array_equal(res[i]["density"].view(np.uint32), d.view(np.uint32)), f"density {i}"
        assert np.array_equal(res[i]["cells"].view(np.uint32), c.view(np.uint32)), f"cells {i}"
        assert np.array_equal(res[i]["pos64"].view(np.uint64), p.view(np.uint64)), f"masters {i}"
