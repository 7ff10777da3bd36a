"""The benchmark configurations at their stated sizes, checked on the GPU through the C ABI.

* n = 20 plain method (graph state on G(20, 1/2), a random single-qubit Clifford per qubit, a U3 layer; order of
  width <= 10): amplitudes of 1,024 uniform random bitstrings and 100 exact chain-rule samples against a brute-force
  2^20 statevector, as the reference's own tests check small circuits against dense states (test_amp.py).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gnp20():
    import workloads
    from oracle import statevector
    w = workloads.graph_state_instance(20, 0.5, seed=1)
    p = statevector.probabilities(20, list(w["body"]) + list(w["tail"]))
    return w, p


def _index(w, string):
    """statevector index of a step-order string (qubit 0 most significant)."""
    by_q = [0] * w["n"]
    for k, st in enumerate(w["steps"]):
        by_q[st["v"]] = int(string[k])
    idx = 0
    for b in by_q:
        idx = 2 * idx + b
    return idx


@pytest.mark.parametrize("prec", [128, 64])
def test_config1_amplitudes_and_samples_vs_statevector(gnp20, prec):
    """1,024 uniform strings: |d Pr| <= 1e-12 (complex128) / 1e-8 (complex64) and |d log2 Pr| <= 1e-9 / 1e-5 where
    Pr > 1e-10; 100 exact samples: each sample's log2 Pr is the statevector's, and its bits equal the oracle's
    sample for the same seed (the reference's mt19937_64 stream)."""
    import os
    import tempfile
    import gsb
    import workloads
    from oracle import Oracle
    w, p = gnp20
    assert w["width"] <= 10
    ns = len(w["steps"])
    strings = workloads.random_strings(ns, 1024, seed=2024)
    ref = np.array([p[_index(w, s)] for s in strings])
    tol_p, tol_lp = (1e-12, 1e-9) if prec == 128 else (1e-8, 1e-5)
    with gsb.Engine.from_text(w["plan"], precision=prec) as eng:
        lp, cond = eng.chain(strings)
        bits, slp = eng.sample(100, 777)
    assert np.abs(np.exp2(lp) - ref).max() <= tol_p
    big = ref > 1e-10
    assert big.sum() >= 1000 and np.abs(lp[big] - np.log2(ref[big])).max() <= tol_lp
    # the conditionals multiply out to the probability
    assert np.abs(np.log2(np.prod(cond, axis=1)) - lp).max() <= (1e-9 if prec == 128 else 1e-5)
    sref = np.array([p[_index(w, b)] for b in bits])
    assert (sref > 0).all() and np.abs(slp - np.log2(sref)).max() <= tol_lp
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "plan.txt")
        open(path, "w").write(w["plan"])
        orc = Oracle(path, prec)
        for i in range(100):
            obits, _ = orc.sample(0, 777, i)
            assert list(bits[i]) == list(obits), i
        orc.close()
