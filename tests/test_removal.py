"""Dead-cell compaction without a GPU: the oracle's restatement of phase 3 of
updatePhenotypes over CellData::removeCell against the reference's own
code (the committed fixture, and the live reference library when it was
built), and the library's host-only move list (pcg_removal_plan) against
the oracle."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def random_case(rng, with_repeats):
    mc = int(rng.integers(1, 70))
    n = int(rng.integers(0, mc + 1))
    S = int(rng.integers(0, 4))
    soa = rng.standard_normal(28 * mc).astype(np.float32)
    soa[23 * mc:28 * mc] = rng.integers(0, 1 << 30, 5 * mc).astype(np.uint32).view(np.float32)
    rates = [rng.standard_normal(max(mc * S, 1)) for _ in range(4)]
    active = rng.integers(0, 2, mc).astype(np.uint8)
    if with_repeats:   # repeats and indices at or past the count
        idx = rng.integers(0, n + 4, int(rng.integers(0, n + 4))).astype(np.uint32)
    else:
        idx = rng.choice(max(n, 1), int(rng.integers(0, n + 1)), replace=False).astype(np.uint32)
    return mc, n, S, soa, rates, active, idx


def test_oracle_matches_reference_fixture(po):
    d = np.load(os.path.join(GOLDEN, "removal.npz"))
    mc, n, S = int(d["max_cells"]), int(d["n"]), int(d["S"])
    soa = d["soa0"].copy()
    rates = [d[k + "0"].copy() for k in ("sec", "upt", "sat", "ne")]
    n_final = po.cells_remove(soa, mc, n, S, *rates, None, d["indices"])
    assert n_final == int(d["n_final"])
    assert np.array_equal(soa.view(np.uint32), d["soa"].view(np.uint32))
    for got, k in zip(rates, ("sec", "upt", "sat", "ne")):
        assert np.array_equal(got, d[k])


@pytest.mark.parametrize("with_repeats", [False, True], ids=["distinct", "repeats"])
def test_oracle_matches_live_reference(po, with_repeats):
    if not po.ref_available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(41 + with_repeats)
    for _ in range(200):
        mc, n, S, soa, rates, active, idx = random_case(rng, with_repeats)
        a_soa, a_rates = soa.copy(), [r.copy() for r in rates]
        b_soa, b_rates = soa.copy(), [r.copy() for r in rates]
        na = po.cells_remove(a_soa, mc, n, S, *a_rates, active.copy(), idx)
        nb = po.ref_cells_remove(b_soa, mc, n, S, *b_rates, idx)
        assert na == nb
        assert np.array_equal(a_soa.view(np.uint32), b_soa.view(np.uint32))
        for x, y in zip(a_rates, b_rates):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("with_repeats", [False, True], ids=["distinct", "repeats"])
def test_removal_plan_reproduces_oracle(pcg, po, with_repeats):
    """Applying pcg_removal_plan's moves (destinations below the new count,
    sources at or past it) gives the oracle's compacted arrays."""
    rng = np.random.default_rng(53 + with_repeats)
    for _ in range(300):
        mc, n, S, soa, rates, active, idx = random_case(rng, with_repeats)
        want_soa, want_rates, want_act = soa.copy(), [r.copy() for r in rates], active.copy()
        n_final = po.cells_remove(want_soa, mc, n, S, *want_rates, want_act, idx)
        dest, src, nf = pcg.removal_plan(n, idx)
        assert nf == n_final
        assert np.all(dest < nf) and np.all(src >= nf) and np.all(src < max(n, 1))
        assert len(set(dest.tolist())) == len(dest)
        got = soa.reshape(28, mc).copy()
        got[:, dest] = got[:, src]
        assert np.array_equal(got[:, :nf].view(np.uint32), want_soa.reshape(28, mc)[:, :nf].view(np.uint32))
        for r, w in zip(rates, want_rates):
            g = r[:mc * S].reshape(mc, S).copy() if S else r[:0]
            if S:
                g[dest] = g[src]
                assert np.array_equal(g[:nf], w[:mc * S].reshape(mc, S)[:nf])
        a = active.copy()
        a[dest] = a[src]
        assert np.array_equal(a[:nf], want_act[:nf])


def test_removal_plan_edge_cases(pcg):
    """Nothing to remove, an empty store, everything removed, indices all
    past the count."""
    assert pcg.removal_plan(0, [])[2] == 0
    d, s, nf = pcg.removal_plan(5, [])
    assert nf == 5 and len(d) == 0 and len(s) == 0
    d, s, nf = pcg.removal_plan(0, [0, 3])
    assert nf == 0 and len(d) == 0
    d, s, nf = pcg.removal_plan(4, [3, 1, 0, 2])
    assert nf == 0 and len(d) == 0
    d, s, nf = pcg.removal_plan(4, [4, 9, 100])
    assert nf == 4 and len(d) == 0
    d, s, nf = pcg.removal_plan(4, [0])
    assert nf == 3 and d.tolist() == [0] and s.tolist() == [3]
