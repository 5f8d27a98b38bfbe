"""pcg_sort_pairs_static — the binning sort on caller-owned device buffers
with static scratch, no device allocation — against the same sort inside
pcg_mech_forces, read back with pcg_mech_bins: sorting the cells'
mechanics-voxel keys with their indices as values gives the cell order of
the existing entry point, bit for bit, on two consecutive calls.

Named to be collected last, so it also runs after every other GPU test has
used (and freed) device memory in the same process.  One case runs in a
fresh process, where no mechanics step has loaded the sort's kernels: after
the set-up call, a sort makes no library allocation and leaves the device's
free memory unchanged."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PCG_ERR_INVALID = 1               # include/pcg.h
MAX_PAIRS = 1 << 18               # PCG_SORT_STATIC_MAX_PAIRS


def _cells(pcg, ctx, n, seed):
    rng = np.random.default_rng(seed)
    soa = np.zeros(28 * n, np.float32)
    pos = rng.random((n, 3)) * 600.0
    for a in range(3):
        soa[a * n:(a + 1) * n] = pos[:, a]
    soa[9 * n:10 * n] = 8.41
    soa[11 * n:12 * n] = 2494.0
    soa[13 * n:14 * n] = 10.0
    soa[14 * n:15 * n] = 0.4
    soa[15 * n:16 * n] = 1.25
    cells = pcg.Cells(ctx, n, 1)
    cells.upload(soa, n, n)
    mp = pcg.mech_params_for_domain(0.0, 600.0, 0.0, 600.0, 0.0, 600.0, False, 0.1)
    mech = pcg.CellMechanics(ctx, mp, (0.0, 0.0, 0.0), n)
    mech.computeForces(cells)
    keys = cells.download(n)[27 * n:28 * n].view(np.uint32).copy()
    _, order = mech.syncHashPointers(n)
    return keys, order, mech.totalMechVoxels()


def _static_sort(pcg, ctx, torch, kd, vd, ko, vo, n, bits):
    torch.cuda.synchronize()
    ctx.check(pcg.lib().pcg_sort_pairs_static(ctx.h, kd.data_ptr(), vd.data_ptr(), ko.data_ptr(), vo.data_ptr(),
                                              n, bits))
    ctx.sync()
    return ko.cpu().numpy().view(np.uint32).copy(), vo.cpu().numpy().view(np.uint32).copy()


@pytest.mark.parametrize("n", [1, 2047, 60000, MAX_PAIRS])
def test_static_sort_matches_mechanics_binning(ctx, pcg, n):
    torch = pytest.importorskip("torch")
    ctx.check(pcg.lib().pcg_sort_pairs_static(ctx.h, None, None, None, None, 0, 32))   # set-up call
    keys, order, tmv = _cells(pcg, ctx, n, 7 + n)
    bits = max(1, int(np.ceil(np.log2(max(tmv, 2)))))
    kd = torch.from_numpy(keys.view(np.int32)).cuda()
    vd = torch.arange(n, dtype=torch.int32, device="cuda")
    ko = torch.empty_like(kd)
    vo = torch.empty_like(vd)
    for b in (bits, 32):
        for _ in range(2):   # two consecutive calls reuse the same static scratch
            ks, vs = _static_sort(pcg, ctx, torch, kd, vd, ko, vo, n, b)
            assert np.array_equal(vs, order)
            assert np.array_equal(ks, keys[order])
            ko.fill_(-1)
            vo.fill_(-1)


@pytest.mark.parametrize("n", [31, 2048, 2049, 100_003, MAX_PAIRS])
@pytest.mark.parametrize("kind", ["equal", "descending", "random32", "top_digit", "few"])
def test_static_sort_key_patterns(ctx, pcg, n, kind):
    """Stable order (numpy's stable argsort) for key patterns that stress the
    per-digit look-back: one key, descending keys, full 32-bit keys, keys
    that differ only in the top digit and a handful of distinct keys."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(n + len(kind))
    keys = {"equal": np.full(n, 0xABCDE, np.uint32),
            "descending": np.arange(n, 0, -1, dtype=np.uint32) * 977,
            "random32": rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32),
            "top_digit": (rng.integers(0, 256, n).astype(np.uint32) << 24) | 0x00123456,
            "few": rng.choice(np.array([3, 70000, 1 << 31, 5], np.uint32), n)}[kind]
    kd = torch.from_numpy(keys.view(np.int32)).cuda()
    vd = torch.arange(n, dtype=torch.int32, device="cuda")
    ko, vo = torch.empty_like(kd), torch.empty_like(vd)
    ks, vs = _static_sort(pcg, ctx, torch, kd, vd, ko, vo, n, 32)
    order = np.argsort(keys, kind="stable").astype(np.uint32)
    assert np.array_equal(vs, order)
    assert np.array_equal(ks, keys[order])


FRESH = textwrap.dedent("""
    import ctypes as C, importlib.util, os, sys
    import numpy as np
    import torch
    pkg = sys.argv[1]
    spec = importlib.util.spec_from_file_location("pcg", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    pcg = importlib.util.module_from_spec(spec); sys.modules["pcg"] = pcg; spec.loader.exec_module(pcg)
    L = pcg.lib()
    ctx = pcg.Context(0)
    ctx.check(L.pcg_sort_pairs_static(ctx.h, None, None, None, None, 0, 32))    # set-up call
    n = 60000
    rng = np.random.default_rng(5)
    keys = rng.integers(0, 1 << 20, n).astype(np.uint32)
    kd = torch.from_numpy(keys.view(np.int32)).cuda()
    vd = torch.arange(n, dtype=torch.int32, device="cuda")
    ko, vo = torch.empty_like(kd), torch.empty_like(vd)
    torch.cuda.synchronize()
    m0, r0 = C.c_uint64(), C.c_uint64()
    L.pcg_debug_alloc_stats(C.byref(m0), C.byref(r0))
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        ctx.check(L.pcg_sort_pairs_static(ctx.h, kd.data_ptr(), vd.data_ptr(), ko.data_ptr(), vo.data_ptr(), n, 20))
        ctx.sync()
    free1 = torch.cuda.mem_get_info()[0]
    m1, r1 = C.c_uint64(), C.c_uint64()
    L.pcg_debug_alloc_stats(C.byref(m1), C.byref(r1))
    order = np.argsort(keys, kind="stable").astype(np.uint32)
    assert np.array_equal(vo.cpu().numpy().view(np.uint32), order)
    assert np.array_equal(ko.cpu().numpy().view(np.uint32), keys[order])
    assert (m1.value, r1.value) == (m0.value, r0.value), ((m0.value, r0.value), (m1.value, r1.value))
    assert free1 == free0, (free0, free1)
    ctx.close()
    print("fresh ok")
""")


def test_fresh_process_sort_allocates_nothing(pcg, tmp_path):
    """In a process where nothing but the set-up call has run, two sorts make
    no library allocation and the device's free memory does not change."""
    pytest.importorskip("torch")
    script = tmp_path / "fresh_sort.py"
    script.write_text(FRESH)
    pkg = os.path.dirname(pcg.__file__)
    res = subprocess.run([sys.executable, str(script), pkg], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "fresh ok" in res.stdout


def test_static_sort_rejects_oversize_and_overlap(ctx, pcg):
    torch = pytest.importorskip("torch")
    lim = MAX_PAIRS
    buf = torch.zeros(4, 8, dtype=torch.int32, device="cuda")
    p = [buf[i].data_ptr() for i in range(4)]
    st = pcg.lib().pcg_sort_pairs_static(ctx.h, p[0], p[1], p[2], p[3], lim + 1, 32)
    assert st == PCG_ERR_INVALID
    assert b"static limit" in pcg.lib().pcg_last_error_string(ctx.h)
    assert pcg.lib().pcg_sort_pairs_static(ctx.h, p[0], p[1], p[0], p[3], 8, 32) == PCG_ERR_INVALID
    assert pcg.lib().pcg_sort_pairs_static(ctx.h, p[0], p[1], p[2], p[3], 8, 0) == PCG_ERR_INVALID
    ctx.sync()
