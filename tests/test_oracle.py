"""Pin the oracle before trusting it (CPU only): the C restatement of the reference executor must reproduce the
reference executor's own outputs (compiled from its sources, recorded in tests/golden/executor_cases.json) and the
reference's published vectors (random streams, the width-30 gate values)."""
import json
import math
import os
import tempfile

import numpy as np
import pytest

from conftest import parse_ref_lines


def _lines(path):
    return [ln.rstrip("\n") for ln in open(path) if ln.strip()]


def test_random_stream_matches_rngbits(w30_dir):
    """results/rngbits_seeds_2000000.txt: bit U < 0.5 of 70 draws of mt19937_64(seed) (rngbits.cpp)."""
    from oracle import uniforms
    for ln in _lines(os.path.join(w30_dir, "rngbits_2000000.txt")):
        bits, seed = ln.split()
        u = uniforms(0, int(seed), 0, 70)
        assert "".join("1" if x < 0.5 else "0" for x in u) == bits


def _close(a, b, tol, ptol):
    if math.isinf(a) and math.isinf(b):
        return True
    return abs(a - b) <= tol or (max(a, b) < -20 and abs(2.0 ** a - 2.0 ** b) <= ptol)


@pytest.mark.parametrize("prec", [128, 64])
def test_oracle_vs_reference_executor(executor_cases, planner_cases, prec):
    from oracle import Oracle
    tol, ptol, ctol = (1e-9, 1e-12, 1e-9) if prec == 128 else (1e-5, 1e-7, 1e-6)
    texts = {c["name"]: c["inplace_plan"] for c in planner_cases["cases"]}
    with tempfile.TemporaryDirectory() as td:
        for ec in executor_cases:
            path = os.path.join(td, "p.txt")
            open(path, "w").write(texts[ec["name"]])
            o = Oracle(path, prec)
            for s, ref in zip(ec["strings"], ec[f"prob{prec}"]):
                assert _close(o.prob(s), float(ref), tol, ptol)
            for s, row in zip(ec["strings"], parse_ref_lines(ec[f"chain{prec}"])):
                lp, cond = o.chain1(s)
                assert _close(lp, float(row[0]), tol, ptol)
                assert np.abs(cond - np.array([float(x) for x in row[1:]])).max() <= ctol
            for key, mode, seed in ((f"sample{prec}", 0, 1000), (f"sample2_{prec}", 1, 5)):
                for i, row in enumerate(parse_ref_lines(ec[key])):
                    bits, lp = o.sample(mode, seed, i)
                    assert "".join(map(str, bits)) == row[0]
                    assert _close(lp, float(row[1]), tol, ptol)
            for li, (line, row) in enumerate(zip(ec["hybrid_lines"], parse_ref_lines(ec[f"hybrid{prec}"]))):
                bits, lp, cond = o.hybrid(line, 9, li)
                assert "".join(map(str, bits)) == row[0]
                assert _close(lp, float(row[1]), tol, ptol)
                assert np.abs(cond - np.array([float(x) for x in row[2:]])).max() <= ctol
            K = ec["K"]
            for li, (line, prow, rrow) in enumerate(zip(ec["prefix_lines"], parse_ref_lines(ec[f"prefix{prec}"]),
                                                         parse_ref_lines(ec[f"resume{prec}"]))):
                dump, ls, lp = o.prefix(line, K)
                assert _close(lp, float(prow[1]), tol, ptol) and abs(ls - float(prow[2])) <= 1e-6
                bits, lpf, lpp, cond = o.resume(line, K, 3, li, [dump], [ls])
                assert "".join(map(str, bits)) == rrow[0]
                assert _close(lpf, float(rrow[1]), tol, ptol) and _close(lpp, float(rrow[2]), tol, ptol)
                assert np.abs(cond[K:] - np.array([float(x) for x in rrow[3:]])).max() <= ctol
            o.close()


def test_oracle_sliced_sum_is_linear(executor_cases, planner_cases):
    """resume over two dumps that are halves of one table (d/2 + d/2, equal logscales) equals resume over d; a twist
    translation by zero is the identity; a bad twist is the reference's exit code 14."""
    from oracle import Oracle
    texts = {c["name"]: c["inplace_plan"] for c in planner_cases["cases"]}
    ec = executor_cases[3]
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "p.txt")
        open(path, "w").write(texts[ec["name"]])
        o = Oracle(path, 128)
        K = ec["K"]
        line = ec["prefix_lines"][0]
        d, ls, _ = o.prefix(line, K)
        a = o.resume(line, K, 3, 0, [d], [ls])
        b = o.resume(line, K, 3, 0, [d / 2, d / 2], [ls, ls])
        c = o.resume(line, K, 3, 0, [d / 2, d / 2], [ls, ls], twist=[(0, 0), (0, 0)])
        assert "".join(map(str, a[0])) == "".join(map(str, b[0])) == "".join(map(str, c[0]))
        assert abs(a[1] - b[1]) < 1e-12 and abs(a[1] - c[1]) < 1e-12
        nk, _ = o.dump_shape(K)
        with pytest.raises(ValueError):
            o.resume(line, K, 3, 0, [d], [ls], twist=[(1 << nk, 0)])


def test_oracle_width30_gate(w30_dir):
    """The C oracle (complex64, one pass per step) on the first width-30 gate string reproduces the gate value of
    cloud_ibmxeb/run.sh:19-21 within 1e-5, and the reference executor's own chain output."""
    from oracle import Oracle
    gate = json.load(open(os.path.join(w30_dir, "gate_log2p.json")))
    s = _lines(os.path.join(w30_dir, "gate_strings.txt"))[0]
    o = Oracle(os.path.join(w30_dir, "nq70_inplace_plan.txt"), 64)
    lp, cond = o.chain1(s)
    o.close()
    assert abs(lp - gate["log2p"][0]) <= gate["tol"]
    ref_path = os.path.join(w30_dir, "gate_ref_outputs.json")
    if os.path.exists(ref_path):
        row = [float(x) for x in json.load(open(ref_path))["chain64"][0].split()]
        assert abs(lp - row[0]) <= 1e-6 and np.abs(cond - np.array(row[1:])).max() <= 1e-7
