"""Failure detection of the fused passes' bounded waits, without a GPU fault.

The test hook withholds the passes' tile loads, so the mbarrier every CTA waits on never completes: each wait gives
up after its limit (about a second), the kernel records the failure in device state and returns, and the host call
reports GSB_E_CUDA.  Nothing traps or hangs.  The engine must then still be usable: with the hook off, the same
strings give the oracle's results.
"""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wide_case():
    import workloads
    w = workloads.matching_instance(38, 38, 7, 8, 20000)
    path = os.path.join(tempfile.mkdtemp(), "plan.txt")
    open(path, "w").write(w["plan"])
    w["path"] = path
    return w


@pytest.mark.parametrize("partial", [False, True])
def test_bounded_wait_runs_out_and_is_reported(wide_case, partial):
    """partial=False starves every CTA of a fused pass; partial=True only the odd ones, so the other CTAs finish
    their tiles and meet the failed ones in the grid reduction's block count."""
    import gsb
    import workloads
    from oracle import Oracle
    ns = len(wide_case["steps"])
    strings = workloads.random_strings(ns, 2, seed=7)
    o = Oracle(wide_case["path"], 128)
    ref = [o.chain1(s)[0] for s in strings]
    o.close()
    with gsb.Engine(wide_case["path"], precision=gsb.GSB_C128) as eng:
        eng.set_fusion(2)
        assert max(eng.fusion_groups()[0]) >= 2          # the plan has fused passes to starve
        eng.test_withhold_tile_loads(True, partial=partial)
        with pytest.raises(gsb.GsbError) as e:
            eng.chain(strings[:1])
        assert e.value.code == 20 and "gave up waiting" in str(e.value)
        eng.test_withhold_tile_loads(False)
        lp, _ = eng.chain(strings)
        assert np.max(np.abs(lp - np.array(ref))) <= 1e-9
        bits, slp = eng.sample(2, 31)                   # the sampling passes use the same reduction
        o = Oracle(wide_case["path"], 128)
        for i in range(2):
            ob, olp = o.sample(0, 31, i)
            assert list(bits[i]) == list(ob) and abs(slp[i] - olp) <= 1e-9
        o.close()
