"""Object lifetimes across the C ABI: a context stays alive while objects made
on it exist, so they may be destroyed in any order, and a script that leaves
them open at interpreter exit (where Python finalises objects held in
reference cycles in no fixed order) exits cleanly."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_context_closed_before_its_batch(pcg):
    from pcg import workloads
    insts = workloads.batched_3d(n_instances=3, seed=11)
    ref_ctx = pcg.Context(0)
    ref = pcg.Batch(ref_ctx, insts)
    ref.step(4)
    ref_ctx.sync()
    want = [ref.density(i) for i in range(len(insts))]
    ref.close()
    ref_ctx.close()

    c = pcg.Context(0)
    b = pcg.Batch(c, insts)
    me = pcg.Microenvironment(c, pcg.make_grid(8, 8, 1, 1), pcg.make_substrates([(1e5, 0.1, True, 38.0)]))
    srv = pcg.Server(c)
    c.close()            # the owner's reference goes first
    b.step(4)            # the batch still holds the context
    got = [b.density(i) for i in range(len(insts))]
    for w, g in zip(want, got):
        np.testing.assert_array_equal(w, g)
    srv.close()
    me.close()
    b.close()            # the last reference frees the context


def test_objects_left_open_at_exit(tmp_path):
    script = tmp_path / "left_open.py"
    script.write_text(textwrap.dedent(f"""
        import faulthandler, importlib.util, sys
        faulthandler.enable()
        pkg = {os.path.join(ROOT, "physicell-mac-metal_b200")!r}
        spec = importlib.util.spec_from_file_location("pcg", pkg + "/__init__.py",
                                                      submodule_search_locations=[pkg])
        pcg = importlib.util.module_from_spec(spec)
        sys.modules["pcg"] = pcg
        spec.loader.exec_module(pcg)
        from pcg import workloads

        def period(batches):          # a function here ties the module's dict into a cycle
            for b in batches:
                b.step(10)

        insts = workloads.batched_3d(n_instances=6, seed=3)
        ctxs = [pcg.Context(0) for _ in range(3)]
        batches = [pcg.Batch(ctxs[k], insts[2 * k:2 * k + 2]) for k in range(3)]
        srv = pcg.Server(ctxs[0])
        period(batches)
        for c in ctxs:
            c.sync()
        print("done", flush=True)
    """))
    r = subprocess.run([sys.executable, str(script)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "done" in r.stdout
