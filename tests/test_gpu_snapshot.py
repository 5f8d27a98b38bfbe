"""Asynchronous .mat snapshots (pcg_snapshot_*) against the reference's own
writer (writeMatlabSnapshots, src/output_writer.cpp:295-452): the files
must be byte-identical to the golden files the reference wrote for the same
cells and density (tests/golden/matlab_*.npz), and a snapshot must capture
the state at the moment it was taken even when the simulation steps on
right after it."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _setup(pcg, ctx, f):
    grid, geo = f["grid"], f["geo"]
    g = pcg.make_grid(int(grid[0]), int(grid[1]), int(grid[2]), int(grid[3]), dx=float(geo[0]), dt=float(geo[3]),
                      x_min=float(geo[4]), y_min=float(geo[5]), z_min=float(geo[6]), dy=float(geo[1]), dz=float(geo[2]))
    S = int(grid[3])
    me = pcg.Microenvironment(ctx, g, pcg.make_substrates([(1e4, 0.1, True, 5.0)] * S))
    me.setDensityAll(f["density"])
    n, mc = int(f["n"]), int(f["max_cells"])
    cells = pcg.Cells(ctx, mc, S)
    cells.upload(f["soa"], n, mc)
    cells.set_secretion(f["sec"], f["upt"], f["sat"], f["ne"])
    return me, cells


@pytest.mark.parametrize("name", ["matlab_2d", "matlab_3d"])
def test_frame_is_byte_identical_to_reference_writer(ctx, pcg, name, tmp_path):
    f = np.load(os.path.join(GOLDEN, name + ".npz"))
    me, cells = _setup(pcg, ctx, f)
    snap = pcg.Snapshot(ctx)
    snap.frame(me, cells, tmp_path, 3, n_cell_types=int(f["n_types"]))
    snap.wait()
    got_cells = open(tmp_path / "output00000003_cells.mat", "rb").read()
    got_env = open(tmp_path / "output00000003_microenvironment0.mat", "rb").read()
    assert got_cells == f["cells_mat"].tobytes()
    assert got_env == f["env_mat"].tobytes()
    for x in (snap, cells, me):
        x.close()


def test_snapshot_is_taken_before_later_steps(ctx, pcg, po, tmp_path):
    f = np.load(os.path.join(GOLDEN, "matlab_3d.npz"))
    me, cells = _setup(pcg, ctx, f)
    before = me.densityBuffer().copy()
    snap = pcg.Snapshot(ctx)
    snap.microenvironment(me, tmp_path / "env.mat")
    me.simulateDiffusionDecay(20)          # queued right behind the snapshot
    snap.wait()
    ctx.sync()
    name, m = po.read_mat4(str(tmp_path / "env.mat"))
    S = int(f["grid"][3])
    nv = before.size // S
    assert name == "multiscale_microenvironment" and m.shape == (4 + S, nv)
    for s in range(S):
        assert np.array_equal(m[4 + s], before[s * nv:(s + 1) * nv].astype(np.float64))
    assert not np.array_equal(me.densityBuffer(), before)   # the simulation did move on
    for x in (snap, cells, me):
        x.close()


def test_unwritable_path_is_reported(ctx, pcg, tmp_path):
    f = np.load(os.path.join(GOLDEN, "matlab_2d.npz"))
    me, cells = _setup(pcg, ctx, f)
    snap = pcg.Snapshot(ctx)
    snap.microenvironment(me, tmp_path / "no_such_dir" / "env.mat")
    with pytest.raises(pcg.PcgError):
        snap.wait()
    snap.wait()                             # the failure is reported once
    for x in (snap, cells, me):
        x.close()
