"""Batched and served simulations: every instance's result is bit-for-bit
what it gets when it runs alone, and alone it matches the oracle."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_mix(pcg, seed=5):
    """Uneven 2-D and 3-D instances with cells."""
    from pcg import workloads
    out = []
    rng = np.random.default_rng(seed)
    for i, (side, nz) in enumerate([(37, 1), (20, 20), (64, 1), (33, 29), (50, 1), (41, 41)]):
        S = 1 + i % 3
        two_d = nz == 1
        g = pcg.make_grid(side, side, nz, S, dx=20.0, dt=0.01, z_min=-10.0 if two_d else 0.0)
        subs = [(1e5, 0.1, True, 38.0)] + [(float(rng.uniform(1e3, 5e4)), float(rng.uniform(0, 0.5)),
                                            bool(rng.integers(0, 2)), 2.0) for _ in range(S - 1)]
        L = side * 20.0
        n = int(rng.integers(50, 3000))
        if two_d:
            pos = np.stack([rng.uniform(0, L, n), rng.uniform(0, L, n), np.zeros(n)], 1).astype(np.float32)
        else:
            pos = rng.uniform(0.3 * L, 0.7 * L, (n, 3)).astype(np.float32)
        out.append(workloads.instance(g, subs, pos, np.full(n, 8.41, np.float32), float(rng.uniform(5, 20)),
                                      float(rng.uniform(0, 1)), 1.25, sec=rng.uniform(0, 5, n * S),
                                      upt=rng.uniform(0, 10, n * S), sat=rng.uniform(0, 40, n * S),
                                      ne=rng.uniform(-5, 5, n * S), two_d=two_d,
                                      flags=pcg.INST_REFRESH_VOXELS if i % 2 else 0))
    return out


def run_batch(pcg, ctx, insts, steps, **kw):
    b = pcg.Batch(ctx, insts, **kw)
    b.step(steps)
    ctx.sync()
    res = [(b.density(i), b.cells(i)) for i in range(len(insts))]
    b.close()
    return res


def test_batch_equals_alone_bitwise(ctx, pcg):
    insts = small_mix(pcg)
    steps = 23   # includes two mechanics steps
    together = run_batch(pcg, ctx, insts, steps)
    for i, inst in enumerate(insts):
        alone = run_batch(pcg, ctx, [inst], steps)[0]
        assert np.array_equal(together[i][0].view(np.uint32), alone[0].view(np.uint32)), f"density {i}"
        assert np.array_equal(together[i][1].view(np.uint32), alone[1].view(np.uint32)), f"cells {i}"


def test_graphs_equal_direct_launches(ctx, pcg):
    insts = small_mix(pcg, seed=6)
    a = run_batch(pcg, ctx, insts, 21, use_graphs=True)
    b = run_batch(pcg, ctx, insts, 21, use_graphs=False, autotune=False)
    for (da, ca), (db, cb) in zip(a, b):
        assert np.array_equal(da.view(np.uint32), db.view(np.uint32))
        assert np.array_equal(ca.view(np.uint32), cb.view(np.uint32))


def test_period_graph_equals_single_steps(ctx, pcg):
    """A call covering whole mechanics periods launches each as one graph;
    the result is the same bits as one sub-step per call, with the same
    kernel count."""
    insts = small_mix(pcg, seed=14)

    def run(calls):
        b = pcg.Batch(ctx, insts)
        l0 = ctx.launches
        for k in calls:
            b.step(k)
        ctx.sync()
        res = [(b.density(i), b.cells(i)) for i in range(len(insts))]
        n = ctx.launches - l0
        b.close()
        return res, n

    whole, n_whole = run([23])          # two period graphs, then three sub-steps
    single, n_single = run([1] * 23)
    mixed, n_mixed = run([3, 20])       # single sub-steps up to the first firing, then one period graph
    assert n_whole == n_single == n_mixed
    for i in range(len(insts)):
        for other in (single, mixed):
            assert np.array_equal(whole[i][0].view(np.uint32), other[i][0].view(np.uint32)), f"density {i}"
            assert np.array_equal(whole[i][1].view(np.uint32), other[i][1].view(np.uint32)), f"cells {i}"


@pytest.mark.parametrize("pins", [(18, 18), (50, 35), (36, 52), (34, 66)])
def test_pinned_launch_shapes_give_identical_results(ctx, pcg, pins):
    """Warps per CTA and pipeline stages change only the schedule: every
    shape gives the same bits."""
    insts = small_mix(pcg, seed=9)[:4]
    ref = run_batch(pcg, ctx, insts, 13, autotune=False)
    got = run_batch(pcg, ctx, insts, 13, autotune=False, pin_x=pins[0], pin_cols=pins[1])
    for (da, ca), (db, cb) in zip(ref, got):
        assert np.array_equal(da.view(np.uint32), db.view(np.uint32))
        assert np.array_equal(ca.view(np.uint32), cb.view(np.uint32))


def test_plane_pass_equals_separate_sweeps(ctx, pcg):
    """Instances whose x-y planes fit shared memory run the x and y sweeps
    as one pass per plane; the result is the same bits as the separate
    passes, for 2-D (faces in the y pass) and 3-D instances, mixed with
    instances too wide for a plane."""
    from pcg import workloads
    insts = small_mix(pcg, seed=10)
    rng = np.random.default_rng(3)
    for nx, ny, nz in ((300, 40, 1), (260, 30, 12)):       # rows longer than a plane row: tile passes
        g = pcg.make_grid(nx, ny, nz, 2, dx=20.0, dt=0.01, z_min=-10.0 if nz == 1 else 0.0)
        n = 400
        L = np.array([nx, ny, nz]) * 20.0
        pos = (rng.uniform(0.2, 0.8, (n, 3)) * L).astype(np.float32)
        if nz == 1:
            pos[:, 2] = 0.0
        insts.append(workloads.instance(g, [(1e5, 0.1, True, 38.0), (3e3, 0.2, False, 0.0)], pos,
                                        np.full(n, 8.41, np.float32), 10.0, 0.4, 1.25,
                                        sec=rng.uniform(0, 5, 2 * n), upt=rng.uniform(0, 10, 2 * n),
                                        sat=rng.uniform(0, 40, 2 * n), two_d=nz == 1))
    a = run_batch(pcg, ctx, insts, 23, planes=True)
    b = run_batch(pcg, ctx, insts, 23, planes=False)
    for i, ((da, ca), (db, cb)) in enumerate(zip(a, b)):
        assert np.array_equal(da.view(np.uint32), db.view(np.uint32)), f"density {i}"
        assert np.array_equal(ca.view(np.uint32), cb.view(np.uint32)), f"cells {i}"


def test_whole_batch_transfers_pipelined(ctx, pcg):
    """The whole-batch copies run on copy streams through staging buffers:
    three rounds of upload -> steps -> download with no host wait between
    calls give the same bits as with a wait after every call, and the cell
    download is the per-instance downloads side by side."""
    insts = small_mix(pcg, seed=13)
    n_tot = sum(i.n_cells for i in insts)
    runs = []
    for wait in (False, True):
        b = pcg.Batch(ctx, insts)
        arena = b.layout(0)[3]
        up = pcg.PinnedArray((28 * n_tot,))
        outs = [(pcg.PinnedArray((28 * n_tot,)), pcg.PinnedArray((arena,))) for _ in range(3)]
        b.download_all_cells(up.array)
        ctx.sync()
        up.array[3 * n_tot:4 * n_tot] += 0.25          # a host-side velocity change every round
        for k in range(3):
            for call in (lambda: b.upload_all_cells(up.array), lambda: b.step(6 + k),
                         lambda: b.download_all_cells(outs[k][0].array),
                         lambda: b.download_all_density(outs[k][1].array)):
                call()
                if wait:
                    ctx.sync()
        ctx.sync()
        res = [(c.array.copy(), d.array.copy()) for c, d in outs]
        if wait:
            per = [b.cells(i) for i in range(len(insts))]
            whole = np.concatenate([p.reshape(28, -1) for p in per], axis=1).ravel()
            assert np.array_equal(whole.view(np.uint32), res[2][0].view(np.uint32))
        runs.append(res)
        for a in [up] + [x for o in outs for x in o]:
            a.free()
        b.close()
    for k, ((ca, da), (cb, db)) in enumerate(zip(*runs)):
        assert np.array_equal(ca.view(np.uint32), cb.view(np.uint32)), f"cells round {k}"
        assert np.array_equal(da.view(np.uint32), db.view(np.uint32)), f"density round {k}"


def test_masked_cell_download(ctx, pcg):
    """pcg_batch_download_cell_fields: the fields in the mask come back as the
    full download gives them, every other field of the host SoA is left as
    it was; with the steps' field set, a host that keeps the other fields
    holds the whole state."""
    insts = small_mix(pcg, seed=14)
    n_tot = sum(i.n_cells for i in insts)
    b = pcg.Batch(ctx, insts)
    b.step(13)
    full = pcg.PinnedArray((28 * n_tot,))
    part = pcg.PinnedArray((28 * n_tot,))
    b.download_all_cells(full.array)
    ctx.sync()
    for mask in (pcg.STEP_WRITTEN_FIELDS, (1 << 27) | 1, 0b101 << 5):
        part.array[:] = -7.0
        b.download_cell_fields(part.array, mask)
        ctx.sync()
        f = full.array.reshape(28, n_tot)
        q = part.array.reshape(28, n_tot)
        for k in range(28):
            if mask >> k & 1:
                assert np.array_equal(q[k].view(np.uint32), f[k].view(np.uint32)), k
            else:
                assert np.all(q[k] == -7.0), k
    # the fields the steps do not write are those of the upload
    start = np.concatenate([i.soa.reshape(28, -1)[:, :i.n_cells] for i in insts], axis=1)
    f = full.array.reshape(28, n_tot)
    for k in range(28):
        if not (pcg.STEP_WRITTEN_FIELDS >> k & 1):
            assert np.array_equal(f[k].view(np.uint32), start[k].view(np.uint32)), k
    with pytest.raises(pcg.PcgError):
        b.download_cell_fields(part.array, 1 << 28)
    full.free()
    part.free()
    b.close()


def test_masked_cell_upload(ctx, pcg):
    """pcg_batch_upload_cell_fields: the fields in the mask take the host's
    values, every other device field keeps its own; after the host-owned
    fields change (radius, volume and strengths here), stepping gives the
    same bits as a whole upload of the same state."""
    insts = small_mix(pcg, seed=15)
    n_tot = sum(i.n_cells for i in insts)
    runs = []
    for whole in (False, True):
        b = pcg.Batch(ctx, insts)
        b.step(11)
        host = pcg.PinnedArray((28 * n_tot,))
        back = pcg.PinnedArray((28 * n_tot,))
        b.download_all_cells(host.array)
        ctx.sync()
        before = host.array.copy().reshape(28, n_tot)
        h = host.array.reshape(28, n_tot)
        for f in (9, 11, 13, 14):                 # radius, total volume, repulsion, adhesion
            h[f] *= np.float32(1.1)
        h[0] += np.float32(3.0)                   # a field the device owns: must not reach it
        if whole:
            h[0] = before[0]
            b.upload_all_cells(host.array)
        else:
            b.upload_cell_fields(host.array, pcg.HOST_OWNED_FIELDS)
        b.download_all_cells(back.array)
        ctx.sync()
        q = back.array.reshape(28, n_tot)
        for k in range(28):
            want = h[k] if (pcg.HOST_OWNED_FIELDS >> k & 1) else before[k]
            assert np.array_equal(q[k].view(np.uint32), want.view(np.uint32)), k
        b.step(12)
        ctx.sync()
        runs.append([(b.density(i), b.cells(i)) for i in range(len(insts))])
        with pytest.raises(pcg.PcgError):
            b.upload_cell_fields(host.array, 1 << 28)
        host.free()
        back.free()
        b.close()
    for (da, ca), (db, cb) in zip(*runs):
        assert np.array_equal(da.view(np.uint32), db.view(np.uint32))
        assert np.array_equal(ca.view(np.uint32), cb.view(np.uint32))


def test_sweep_units_count_the_passes(ctx, pcg):
    """pcg_batch_sweep_units: with planes a 3-D instance's sub-step moves
    each voxel-substrate twice (x + y plane pass, z plane pass) and a 2-D
    one once, all in plane launches; without planes three and two times."""
    insts = small_mix(pcg, seed=11)
    per_pass = {True: 0, False: 0}          # 3-D?, voxel-substrates
    for inst in insts:
        g = inst.grid
        per_pass[g.nz > 1] += g.nx * g.ny * g.nz * g.n_substrates
    with_planes = 2 * per_pass[True] + per_pass[False]
    for planes, want in ((True, (with_planes, with_planes)), (False, (0, 3 * per_pass[True] + 2 * per_pass[False]))):
        b = pcg.Batch(ctx, insts, autotune=False, planes=planes)
        assert b.sweep_units() == want
        b.close()


@pytest.mark.parametrize("forces,threads", [(256000, 256), (64016, 64), (128032, 128), (256064, 96),
                                            (96000, 160), (32064, 32)])
def test_pinned_cell_kernel_shapes_match_tuned(ctx, pcg, forces, threads, tmp_path):
    """Force pass shapes (threads per block, neighbour queue slots) and the
    block sizes of the secretion, binning and AB2 kernels change no bit:
    every pinned shape gives what the autotuned batch gives, over 23
    sub-steps with two mechanics steps."""
    insts = small_mix(pcg, seed=11)
    tuned = run_batch(pcg, ctx, insts, 23, tune_cache=str(tmp_path / "tune.json"))
    pinned = run_batch(pcg, ctx, insts, 23, autotune=False, pin_forces=forces, pin_cell_threads=threads)
    for (d0, c0), (d1, c1) in zip(tuned, pinned):
        assert np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
        assert np.array_equal(c0.view(np.uint32), c1.view(np.uint32))


def test_tuned_shapes_reported_and_cached(ctx, pcg, tmp_path):
    """The autotuner records its choices for the cell kernels in the tune
    cache and the batch reports them."""
    import json
    cache = tmp_path / "tune.json"
    b = pcg.Batch(ctx, small_mix(pcg, seed=12), tune_cache=str(cache))
    desc = b.describe()
    b.close()
    for k in ("forces(block=", "secrete(block=", "bin(block=", "integrate(block="):
        assert k in desc
    keys = json.loads(cache.read_text()).keys()
    for k in ("forces:", "secrete:", "bin:", "integrate:"):
        assert any(x.startswith(k) for x in keys), (k, list(keys))


@pytest.mark.parametrize("kw", [{"pin_forces": 256000 + 8}, {"pin_forces": 300032}, {"pin_cell_threads": 48},
                                {"pin_cell_threads": 512}])
def test_bad_pinned_cell_shape_is_refused(ctx, pcg, kw):
    with pytest.raises(pcg.PcgError):
        pcg.Batch(ctx, small_mix(pcg, seed=9)[:1], autotune=False, **kw)


def test_bad_pinned_shape_is_refused(ctx, pcg):
    with pytest.raises(pcg.PcgError):
        pcg.Batch(ctx, small_mix(pcg, seed=9)[:1], autotune=False, pin_x=17 * 16 + 2)


def test_batch_instance_matches_oracle(ctx, pcg, po):
    insts = small_mix(pcg, seed=7)
    steps = 31
    res = run_batch(pcg, ctx, insts, steps)
    for i in (0, 1, 3):
        inst = insts[i]
        g = inst.grid
        S, n = g.n_substrates, inst.n_cells
        og = po.make_grid(g.nx, g.ny, g.nz, S, dx=g.dx, dt=g.dt, x_min=g.x_min, y_min=g.y_min, z_min=g.z_min)
        osubs = po.make_subs([(s.diffusion_coefficient, s.decay_rate, bool(s.dirichlet_enabled), s.target_value)
                              for s in inst.substrates[:S]])
        m = inst.mech
        om = po.Mech(m.dt, m.cell_cell_repulsion, m.cell_cell_adhesion, m.max_interaction_distance,
                     m.mechanics_voxel_size, m.mech_grid_nx, m.mech_grid_ny, m.mech_grid_nz)
        dens = np.repeat(inst.initial_values, g.nx * g.ny * g.nz).astype(np.float32)
        soa = inst.soa.copy()
        pm = po.master_positions(soa, n)
        po.run(og, osubs, om, 0.1, dens, soa, n, n, *inst.rates, None, steps, refresh=bool(inst.flags & 1),
               pos64=pm)
        b = np.asarray(dens, np.float64)
        err = np.abs(res[i][0] - b) / np.maximum(np.abs(b), 1e-6 * np.abs(b).max())
        assert err.max() <= 1e-5, (i, err.max())
        assert np.abs(res[i][1][:3 * n].astype(np.float64) - soa[:3 * n]).max() <= 1e-4


def test_upload_cells_between_steps(ctx, pcg):
    insts = small_mix(pcg, seed=8)[:3]
    b = pcg.Batch(ctx, insts)
    b.step(12)
    soa = b.cells(1)
    n = insts[1].n_cells
    soa[3 * n:4 * n] += 1.0          # a host-side velocity change (motility hook)
    b.upload_cells(1, soa, n)
    b.step(10)
    ctx.sync()
    assert np.isfinite(b.density(1)).all()
    b.close()


def test_served_results_equal_alone(ctx, pcg):
    """Continuous batching: requests arrive over several ticks with different
    step counts; each result is bit-for-bit its result alone."""
    insts = small_mix(pcg, seed=9)
    steps = [40, 25, 60, 33, 18, 47]
    srv = pcg.Server(ctx, budget_bytes=int(4e9), steps_per_tick=10)
    ids = []
    for k, (inst, s) in enumerate(zip(insts, steps)):
        ids.append(srv.submit(inst, s))
        srv.tick()                      # arrivals interleave with progress
    for _ in range(200):
        r, q, _ = srv.tick()
        if r == 0 and q == 0:
            break
    for rid, inst, s in zip(ids, insts, steps):
        assert srv.state(rid) == pcg.REQ_DONE
        d, c = srv.fetch(rid)
        alone_d, alone_c = run_batch(pcg, ctx, [inst], s)[0]
        assert np.array_equal(d.view(np.uint32), alone_d.view(np.uint32))
        assert np.array_equal(c.view(np.uint32), alone_c.view(np.uint32))
        t_total, t_run = srv.times(rid)
        assert t_total >= t_run > 0
    v, cs, held = srv.totals()
    assert v > 0 and held == 0
    srv.close()


def test_server_respects_budget(ctx, pcg):
    insts = [small_mix(pcg, seed=10)[3]] * 6          # equal requests: two fit the budget at a time
    one = insts[0].bytes()
    srv = pcg.Server(ctx, budget_bytes=int(one * 2.2), steps_per_tick=5)
    for inst in insts:
        srv.submit(inst, 12)
    peak = 0
    for _ in range(100):
        r, q, _ = srv.tick()
        _, _, held = srv.totals()
        assert held <= one * 2.2
        peak = max(peak, r)
        if r == 0 and q == 0:
            break
    assert peak <= 2
    for rid in srv.requests:
        assert srv.state(rid) == pcg.REQ_DONE
    srv.close()
    tiny = pcg.Server(ctx, budget_bytes=10)
    with pytest.raises(pcg.PcgError):
        tiny.submit(insts[0], 10)          # larger than the whole budget
    tiny.close()


def test_inactive_cells_in_a_batch(ctx, pcg, po):
    """Secretion order with non-secreting cells in every instance (instances
    of one and of two 2048-cell sort tiles): the inactive cells sort after
    each instance's active ones as one run that secretion skips.  Batch and
    alone give the same bits; one instance matches the oracle."""
    insts = small_mix(pcg, seed=9)
    rng = np.random.default_rng(19)
    for inst in insts:
        act = (rng.random(inst.n_cells) < 0.7).astype(np.uint8)
        act[:5] = 0   # inactive cells at the start of the instance's range too
        inst.active = act
    assert any(inst.n_cells > 2048 for inst in insts)
    steps = 23
    together = run_batch(pcg, ctx, insts, steps)
    for i, inst in enumerate(insts):
        alone = run_batch(pcg, ctx, [inst], steps)[0]
        assert np.array_equal(together[i][0].view(np.uint32), alone[0].view(np.uint32)), f"density {i}"
        assert np.array_equal(together[i][1].view(np.uint32), alone[1].view(np.uint32)), f"cells {i}"
    i = max(range(len(insts)), key=lambda k: insts[k].n_cells)
    inst = insts[i]
    g = inst.grid
    S, n = g.n_substrates, inst.n_cells
    og = po.make_grid(g.nx, g.ny, g.nz, S, dx=g.dx, dt=g.dt, x_min=g.x_min, y_min=g.y_min, z_min=g.z_min)
    osubs = po.make_subs([(s.diffusion_coefficient, s.decay_rate, bool(s.dirichlet_enabled), s.target_value)
                          for s in inst.substrates[:S]])
    m = inst.mech
    om = po.Mech(m.dt, m.cell_cell_repulsion, m.cell_cell_adhesion, m.max_interaction_distance,
                 m.mechanics_voxel_size, m.mech_grid_nx, m.mech_grid_ny, m.mech_grid_nz)
    dens = np.repeat(inst.initial_values, g.nx * g.ny * g.nz).astype(np.float32)
    soa = inst.soa.copy()
    pm = po.master_positions(soa, n)
    po.run(og, osubs, om, 0.1, dens, soa, n, n, *inst.rates, inst.active, steps, refresh=bool(inst.flags & 1),
           pos64=pm)
    b = np.asarray(dens, np.float64)
    err = np.abs(together[i][0] - b) / np.maximum(np.abs(b), 1e-6 * np.abs(b).max())
    assert err.max() <= 1e-5, (i, err.max())
