"""updateMotility on the device (pcg_motility_update) against the oracle.

Where the reference's result does not depend on its random draws (bias 1,
persistence below dt) the device must reproduce the reference's own output
bit for bit (the golden fixtures written from src/motility.cpp).  With
random draws both sides use the same counter-based generator: the resample
decisions and elapsed times are exact, the motility vectors agree to 1e-12
of the speed (the double sine and cosine may differ in their last place),
and the velocities to 1e-6 relative."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _me(pcg, ctx, g, dens):
    grid = pcg.make_grid(g.nx, g.ny, g.nz, g.n_substrates, dx=g.dx, dt=g.dt, x_min=g.x_min, y_min=g.y_min,
                         z_min=g.z_min, dy=g.dy, dz=g.dz)
    me = pcg.Microenvironment(ctx, grid, pcg.make_substrates([(1e3, 0.1, False, 0.0)] * g.n_substrates))
    me.setDensityAll(dens)
    return me


def _run_device(pcg, ctx, g, dens, soa, n, mc, st, dt, seeds_steps, layout):
    me = _me(pcg, ctx, g, dens)
    cells = pcg.Cells(ctx, mc, g.n_substrates)
    cells.upload(soa, n, mc)
    mot = pcg.Motility(ctx, mc, st["n_sens"] if st["sensitivity"] is not None else 0)
    mot.upload(st)
    for seed, step in seeds_steps:
        mot.update(cells, me, dt, seed, step, layout)
    ctx.sync()
    out = cells.download(mc)
    el, vec = mot.download()
    for x in (mot, cells, me):
        x.close()
    return out, el, vec


@pytest.mark.parametrize("name", ["motility_2d_legacy", "motility_3d_multi"])
def test_device_matches_reference_golden(ctx, pcg, po, name):
    f = np.load(os.path.join(GOLDEN, name + ".npz"))
    grid, geo = f["grid"], f["geo"]
    g = po.Grid(*[int(x) for x in grid], *[float(x) for x in geo[:4]], *[float(x) for x in geo[4:]], 0.0)
    n, mc, n_sens = int(f["n"]), int(f["max_cells"]), int(f["n_sens"])
    st = po.motility_state(n, n_sens)
    for k in st:
        if isinstance(st[k], np.ndarray):
            st[k] = f["in_" + k].copy()
    soa, el, vec = _run_device(pcg, ctx, g, f["density"], f["soa0"], n, mc, st, 0.1, [(123, 9)], pcg.MOT_REFERENCE)
    assert np.array_equal(vec, f["vec_out"])
    assert np.array_equal(el, f["elapsed_out"])
    ref = f["soa_out"]
    for fld in range(28):   # the n cells held by the store (slots past n are not uploaded)
        assert np.array_equal(soa[fld * mc:fld * mc + n], ref[fld * mc:fld * mc + n]), fld


def _random_case(po, rng, two_d, S, multi, n=2000, mc=2048):
    nx, ny, nz = 30, 24, (1 if two_d else 18)
    g = po.Grid(nx, ny, nz, S, 20.0, 20.0, 20.0, 0.01, -300.0, -240.0, -10.0 if two_d else -180.0, 0.0)
    dens = rng.uniform(0, 40, nx * ny * nz * S).astype(np.float32)
    soa = np.zeros(28 * mc, np.float32)
    soa[0:n] = rng.uniform(-320, 320, n)
    soa[mc:mc + n] = rng.uniform(-260, 260, n)
    soa[2 * mc:2 * mc + n] = 0 if two_d else rng.uniform(-200, 200, n)
    soa[3 * mc:6 * mc] = rng.normal(0, 1, 3 * mc)
    soa[16 * mc:16 * mc + n] = rng.uniform(0.2, 2, n)
    soa[25 * mc:25 * mc + n] = np.where(rng.random(n) < 0.95, 1, 0).astype(np.uint32).view(np.float32)
    st = po.motility_state(n, S if multi else 0)
    st["is_motile"][:] = rng.random(n) < 0.85
    st["persistence_time"][:] = rng.uniform(0.05, 30.0, n)
    st["bias"][:] = rng.uniform(0, 1, n)
    st["restrict_2d"][:] = 1 if two_d else (rng.random(n) < 0.3)
    st["chemotaxis_index"][:] = rng.integers(0, S, n)
    st["chemotaxis_direction"][:] = np.where(rng.random(n) < 0.5, 1, -1)
    if multi:
        st["sensitivity"][:] = np.where(rng.random(n * S) < 0.2, 0.0, rng.uniform(-1, 1, n * S))
    return g, dens, soa, st, n, mc


@pytest.mark.parametrize("two_d,S,multi,layout", [(True, 1, False, 0), (False, 2, True, 0), (False, 3, True, 1),
                                                  (True, 2, False, 1)],
                         ids=["2d_legacy", "3d_multi_ref", "3d_multi_substrate_major", "2d_legacy_substrate_major"])
def test_device_matches_oracle_with_draws(ctx, pcg, po, two_d, S, multi, layout):
    rng = np.random.default_rng(100 + S)
    g, dens, soa, st, n, mc = _random_case(po, rng, two_d, S, multi)
    steps = [(2024, k) for k in range(4)]
    ref_soa = soa.copy()
    ref_st = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    for seed, step in steps:
        po.motility_update(ref_soa, mc, n, dens, g, ref_st, 0.1, seed, step, layout)
    out, el, vec = _run_device(pcg, ctx, g, dens, soa, n, mc, st, 0.1, steps, layout)
    assert np.array_equal(el, ref_st["elapsed"])                       # same resample decisions
    speed = soa[16 * mc:16 * mc + n].astype(np.float64)
    err = np.abs(vec - ref_st["vec"]).reshape(3, n).max(axis=0)
    assert np.all(err <= 1e-12 * np.maximum(speed, 1.0))
    for f in (3, 4, 5):
        a, b = out[f * mc:f * mc + n].astype(np.float64), ref_soa[f * mc:f * mc + n].astype(np.float64)
        assert np.all(np.abs(a - b) <= 1e-6 * (np.abs(b) + 1.0)), f
    others = [f for f in range(28) if f not in (3, 4, 5)]
    assert all(np.array_equal(out[f * mc:(f + 1) * mc], ref_soa[f * mc:(f + 1) * mc]) for f in others)
    dead = soa[25 * mc:25 * mc + n].view(np.uint32) == 0
    assert np.array_equal(out[3 * mc:3 * mc + n][dead], soa[3 * mc:3 * mc + n][dead])   # dead cells untouched


def test_reproducible_and_seed_dependent(ctx, pcg, po):
    rng = np.random.default_rng(9)
    g, dens, soa, st, n, mc = _random_case(po, rng, False, 1, False, n=500, mc=512)
    st["persistence_time"][:] = 0.5
    a = _run_device(pcg, ctx, g, dens, soa, n, mc, {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()},
                    0.1, [(1, 0)], 0)
    b = _run_device(pcg, ctx, g, dens, soa, n, mc, {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()},
                    0.1, [(1, 0)], 0)
    c = _run_device(pcg, ctx, g, dens, soa, n, mc, {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()},
                    0.1, [(2, 0)], 0)
    assert np.array_equal(a[2], b[2]) and not np.array_equal(a[2], c[2])


def test_bad_arguments_are_errors(ctx, pcg):
    mot = pcg.Motility(ctx, 16, 2)
    z = np.zeros(16)
    u = np.zeros(16, np.uint32)
    i = np.zeros(16, np.int32)
    with pytest.raises(pcg.PcgError):   # created with substrates: sensitivity required
        mot.upload({"persistence_time": z, "elapsed": z, "bias": z, "vec": np.zeros(48), "is_motile": u,
                    "restrict_2d": u, "chemotaxis_index": i, "chemotaxis_direction": i, "sensitivity": None})
    with pytest.raises(pcg.PcgError):   # more cells than max_cells
        mot.upload({"persistence_time": np.zeros(17), "elapsed": np.zeros(17), "bias": np.zeros(17),
                    "vec": np.zeros(51), "is_motile": np.zeros(17, np.uint32), "restrict_2d": np.zeros(17, np.uint32),
                    "chemotaxis_index": np.zeros(17, np.int32), "chemotaxis_direction": np.zeros(17, np.int32),
                    "sensitivity": np.zeros(34)})
    mot.close()
