"""Failure detection without a GPU fault.

- Bounded device waits: a test switch makes the first wait of every plane
  CTA report that its bound ran out; the CTA records it, waits (bounded)
  for its own copies and exits.  pcg_sync reports PCG_ERR_DEVICE and the
  context keeps working.  The reference logs a failed command buffer and
  carries on (src/metal_context.mm:448-461).
- Allocation failure, injected on the host: the nth device allocation of
  a batch build fails; the call returns PCG_ERR_OOM, gives back what it had
  taken (a later build needs no new device allocation) and the context
  keeps working.  The reference aborts instead (src/metal_context.mm:52-60).
- Serving: a queued or running request can be cancelled; the others run on
  and give the same results as alone; requests spread over two contexts.
"""
import ctypes as C

import numpy as np
import pytest

from test_gpu_batch import run_batch, small_mix

pytestmark = pytest.mark.gpu

PCG_ERR_INVALID, PCG_ERR_OOM, PCG_ERR_DEVICE = 1, 3, 8      # include/pcg.h


def alloc_stats(pcg):
    m, r = C.c_uint64(), C.c_uint64()
    pcg.lib().pcg_debug_alloc_stats(C.byref(m), C.byref(r))
    return m.value, r.value


def test_wait_that_runs_out_is_reported_and_context_recovers(ctx, pcg):
    insts = small_mix(pcg, seed=21)
    ref = run_batch(pcg, ctx, insts, 5, autotune=False)
    b = pcg.Batch(ctx, insts, autotune=False)
    assert b.sweep_units()[0] > 0                      # the plane kernel runs
    L = pcg.lib()
    ctx.check(L.pcg_debug_give_up_waits(ctx.h, 1))
    try:
        b.step(1)
        st = L.pcg_sync(ctx.h)
    finally:
        ctx.check(L.pcg_debug_give_up_waits(ctx.h, 0))
    assert st == PCG_ERR_DEVICE
    assert b"wait limit" in L.pcg_last_error_string(ctx.h)
    b.close()
    assert L.pcg_sync(ctx.h) == 0                      # reported once, then cleared
    again = run_batch(pcg, ctx, insts, 5, autotune=False)
    for (d0, c0), (d1, c1) in zip(ref, again):
        assert np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
        assert np.array_equal(c0.view(np.uint32), c1.view(np.uint32))


def test_injected_allocation_failure(ctx, pcg):
    insts = small_mix(pcg, seed=22)
    ref = run_batch(pcg, ctx, insts, 12, autotune=False)     # also fills the device pool
    run_batch(pcg, ctx, insts, 1, autotune=False)
    m0, _ = alloc_stats(pcg)
    L = pcg.lib()
    for nth in (1, 2, 7, 20):
        L.pcg_debug_fail_alloc(nth)
        try:
            with pytest.raises(pcg.PcgError) as e:
                pcg.Batch(ctx, insts, autotune=False)
        finally:
            L.pcg_debug_fail_alloc(0)
        assert e.value.status == PCG_ERR_OOM
    # every block the failed builds took went back to the pool: the next
    # build takes them again and makes no new device allocation
    got = run_batch(pcg, ctx, insts, 12, autotune=False)
    assert alloc_stats(pcg)[0] == m0
    for (d0, c0), (d1, c1) in zip(ref, got):
        assert np.array_equal(d0.view(np.uint32), d1.view(np.uint32))
        assert np.array_equal(c0.view(np.uint32), c1.view(np.uint32))
    L.pcg_debug_fail_alloc(1)
    try:
        with pytest.raises(pcg.PcgError) as e:
            pcg.Cells(ctx, 1000, 1)
    finally:
        L.pcg_debug_fail_alloc(0)
    assert e.value.status == PCG_ERR_OOM
    pcg.Cells(ctx, 1000, 1).close()


def test_cancel_queued_and_running_requests(ctx, pcg):
    insts = small_mix(pcg, seed=23)
    steps = [30, 40, 25, 35, 20, 45]
    srv = pcg.Server(ctx, budget_bytes=int(4e9), max_active=3, steps_per_tick=10)
    ids = [srv.submit(inst, s) for inst, s in zip(insts, steps)]
    srv.tick()                                         # three admitted, three queued
    assert [srv.state(r) for r in ids] == [pcg.REQ_RUNNING] * 3 + [pcg.REQ_QUEUED] * 3
    srv.cancel(ids[1])                                 # running
    srv.cancel(ids[4])                                 # queued
    assert srv.state(ids[1]) == pcg.REQ_CANCELLED and srv.state(ids[4]) == pcg.REQ_CANCELLED
    for _ in range(100):
        r, q, _ = srv.tick()
        if r == 0 and q == 0:
            break
    for k, (rid, inst, s) in enumerate(zip(ids, insts, steps)):
        if k in (1, 4):
            assert srv.state(rid) == pcg.REQ_CANCELLED
            with pytest.raises(pcg.PcgError):
                srv.fetch(rid)
            continue
        assert srv.state(rid) == pcg.REQ_DONE
        d, c = srv.fetch(rid)
        alone_d, alone_c = run_batch(pcg, ctx, [inst], s)[0]
        assert np.array_equal(d.view(np.uint32), alone_d.view(np.uint32))
        assert np.array_equal(c.view(np.uint32), alone_c.view(np.uint32))
    with pytest.raises(pcg.PcgError):
        srv.cancel(ids[0])                             # finished
    assert srv.totals()[2] == 0                        # no budget held
    srv.close()


def test_requests_spread_over_two_contexts(ctx, pcg):
    """Two contexts (both on this GPU here; one per GPU in a multi-GPU
    server): each admission goes to the context with the most unused
    budget, each holds at most its budget, and every result is what the
    request gets alone."""
    other = pcg.Context(0)
    insts = small_mix(pcg, seed=24)
    steps = [20, 30, 25, 15, 35, 10]
    per = max(i.bytes() for i in insts) * 2.5
    srv = pcg.Server([ctx, other], budget_bytes=int(per), steps_per_tick=10)
    ids = [srv.submit(inst, s) for inst, s in zip(insts, steps)]
    srv.tick()
    places = [srv.placement(r) for r in ids]
    assert places[0] == 0 and places[1] == 1           # the second goes where the room is
    assert set(p for p in places if p >= 0) == {0, 1}
    for _ in range(200):
        r, q, _ = srv.tick()
        assert srv.totals()[2] <= 2 * per
        if r == 0 and q == 0:
            break
    for rid, inst, s in zip(ids, insts, steps):
        assert srv.state(rid) == pcg.REQ_DONE
        d, c = srv.fetch(rid)
        alone_d, alone_c = run_batch(pcg, ctx, [inst], s)[0]
        assert np.array_equal(d.view(np.uint32), alone_d.view(np.uint32))
        assert np.array_equal(c.view(np.uint32), alone_c.view(np.uint32))
    srv.close()
    other.close()
