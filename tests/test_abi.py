"""The C ABI library without a GPU: it loads, exports every entry point of
include/pcg.h, reports a missing device as an error (no abort), and the
host-side helpers behave."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "pcg.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pcg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(pcg):
    lib = pcg.lib()
    names = declared_symbols()
    assert len(names) > 50
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(pcg.exported_symbols()) == names


def test_abi_version(pcg):
    assert pcg.lib().pcg_abi_version() == 1


def test_struct_layouts_match_reference(pcg):
    """GridParams 48 B, SubstrateParams 32 B, MechanicsParams 32 B (shaders/types.h:23-61)."""
    assert C.sizeof(pcg.GridParams) == 48
    assert C.sizeof(pcg.SubstrateParams) == 32
    assert C.sizeof(pcg.MechanicsParams) == 32


def test_struct_layouts_match_reference_build(pcg, po):
    if not po.ref_available():
        pytest.skip("oracle/_ref not built")
    r = po.ref()
    assert r.ref_sizeof_grid() == C.sizeof(pcg.GridParams)
    assert r.ref_sizeof_substrate() == C.sizeof(pcg.SubstrateParams)
    assert r.ref_sizeof_mech() == C.sizeof(pcg.MechanicsParams)


def test_create_without_device_is_an_error_not_a_crash(pcg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    st = pcg.lib().pcg_create(0, C.byref(h))
    assert st != 0
    assert h.value is None
    with pytest.raises(pcg.PcgError):
        pcg.Context(0)


def test_null_handles_are_rejected(pcg):
    L = pcg.lib()
    assert L.pcg_sync(None) != 0
    assert L.pcg_me_diffuse(None, 1) != 0
    assert L.pcg_mech_forces(None, None) != 0
    assert L.pcg_batch_step(None, 1) != 0
    assert L.pcg_serve_tick(None, None, None, None) != 0
    assert L.pcg_destroy(None) == 0


def test_instance_bytes_host_only(pcg):
    from pcg import workloads
    inst = workloads.plain_2d()
    b = inst.bytes()
    assert 50 * 50 * 4 <= b < 10_000_000


def test_neighbor_hash_matches_oracle(pcg, po):
    for j in (0, 1, 7, 123456, 2 ** 31 + 5):
        assert pcg.lib().pcg_neighbor_hash(j) == po.nbr_hash(j)


def test_mech_grid_rule_matches_oracle(pcg, po):
    for dom in [(-500, 500, -500, 500, -10, 10, True), (0, 3000, 0, 3000, 0, 3000, False),
                (0, 810, 0, 790, 0, 29, False), (-1000, 1000, -1000, 1000, -10, 10, True)]:
        a = pcg.mech_params_for_domain(*dom)
        b = po.mech_params(*dom)
        assert (a.mech_grid_nx, a.mech_grid_ny, a.mech_grid_nz) == (b.mech_grid_nx, b.mech_grid_ny, b.mech_grid_nz)


def test_voxel_index_matches_oracle(pcg, po):
    from pcg import workloads
    g = pcg.make_grid(13, 9, 7, 1, dx=20.0, x_min=-130.0, y_min=-90.0, z_min=0.0)
    rng = np.random.default_rng(3)
    pos = rng.uniform(-200, 200, size=(1000, 3)).astype(np.float32)
    v = workloads.voxel_index(pos[:, 0], pos[:, 1], pos[:, 2], g)
    mc = 1000
    soa = np.zeros(28 * mc, np.float32)
    soa[0:mc], soa[mc:2 * mc], soa[2 * mc:3 * mc] = pos[:, 0], pos[:, 1], pos[:, 2]
    og = po.make_grid(13, 9, 7, 1, dx=20.0, x_min=-130.0, y_min=-90.0, z_min=0.0)
    po.voxel_refresh(soa, mc, mc, og)
    assert np.array_equal(v, soa[26 * mc:27 * mc].view(np.uint32))


def test_workload_shapes(pcg):
    from pcg import workloads
    insts = workloads.batched_3d(n_instances=4)
    for i in insts:
        assert 40 <= i.grid.nx <= 120 and i.grid.nx == i.grid.ny == i.grid.nz
        assert i.grid.n_substrates == 2 and 1000 <= i.n_cells <= 100000
        assert i.mech.mech_grid_nz > 1
    reqs = workloads.serving_requests(horizon_s=2.0)
    assert len(reqs) > 10
    assert all(600 <= s <= 6000 for _, _, s in reqs)
