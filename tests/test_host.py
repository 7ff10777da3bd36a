"""Host-side logic of the executor that needs no GPU: the C ABI's exports, plan parsing and layout validation with
the reference's error codes, the command line's usage errors, the circuit families."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT


def test_library_exports_every_declared_symbol():
    import gsb
    header = open(os.path.join(ROOT, "include", "gsb.h")).read()
    declared = set(re.findall(r"\b(gsb_[a-z0-9_]+)\s*\(", header))
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(gsb.lib(), name), name
    assert declared == set(gsb.EXPORTS)


def test_validator_accepts_planner_output(planner_cases, w30_dir):
    import gsb
    for c in planner_cases["cases"]:
        n, ns, R = gsb.validate_text(c["inplace_plan"])
        assert (n, ns, R) == (c["n"], c["n"], c["R"])
    for f in ("nq70_inplace_plan.txt", "nq70_inplace_plan_regen.txt"):
        assert gsb.validate_text(open(os.path.join(w30_dir, f)).read()) == (70, 70, 30)


def _code(text):
    import gsb
    try:
        gsb.validate_text(text)
    except gsb.GsbError as e:
        return e.code
    return 0


def test_validator_error_codes(planner_cases):
    """Parse failures return the reference's exit codes (gsamp2.cpp:128-135); layout faults return 15."""
    text = [c for c in planner_cases["cases"] if c["n"] >= 6][0]["inplace_plan"]
    lines = text.strip().split("\n")
    assert _code("") == 2
    assert _code("3 x 2") == 2
    assert _code(lines[0] + "\n") == 3                      # steps missing
    toks = lines[2].split()
    nk = int(toks[1])
    assert _code("\n".join(lines[:2] + [" ".join(toks[:6 + max(nk - 1, 0)])])) in (4, 5)
    assert _code("\n".join(lines[:-1] + [" ".join(lines[-1].split()[:-3])])) == 6
    big = toks[:]
    big[1] = "41"
    assert _code("\n".join(lines[:2] + [" ".join(big)] + lines[3:])) == 7
    # a step reading a slot outside the live table: change one Tkeep address to an unused arena bit
    for i in range(2, len(lines)):
        t = lines[i].split()
        if int(t[1]) >= 1:
            R = int(lines[0].split()[2])
            t[6] = str(1 << (R - 1) | int(t[6]))
            bad = "\n".join(lines[:i] + [" ".join(t)] + lines[i + 1:])
            assert _code(bad) == 15
            break
    # a growth slot beyond the 2^R arena (g is read only when m = 2)
    i = next(i for i in range(1, len(lines)) if lines[i].split()[2] == "2")
    t = lines[i].split()
    t[3] = str(1 << 40)
    assert _code("\n".join(lines[:i] + [" ".join(t)] + lines[i + 1:])) == 15


def test_cli_usage_exit_code():
    r = subprocess.run([os.path.join(PKG, "gsb2")], capture_output=True)
    assert r.returncode == 1


def test_cli_bad_plan_exit_code(tmp_path):
    p = tmp_path / "p.txt"
    p.write_text("garbage")
    s = tmp_path / "s.txt"
    s.write_text("0\n")
    r = subprocess.run([os.path.join(PKG, "gsb2"), str(p), "prob", str(s)], capture_output=True)
    from conftest import cuda_available
    # the reference's plan-parse code; a machine without a GPU fails at device set-up first (99)
    assert r.returncode == (2 if cuda_available() else 99)


def test_clifford_group_and_circuits():
    import circuits
    assert len(circuits.CLIFFORD_WORDS) == 24
    n, body, tail = circuits.matching_circuit(9, 4, seed=3)
    czs = [qs for g, qs in body if g == "cz"]
    assert len(czs) == 4 * 4                              # odd n: one idle qubit per layer
    n, body, tail = circuits.graph_state_circuit(8, 0.5, seed=1)
    assert len(tail) == 8 and all(t[0].startswith("u3(") for t in tail)
    import amp
    for name, _ in tail:
        W = amp.gate_matrix(name)
        assert np.allclose(W.conj().T @ W, np.eye(2), atol=1e-14)
    with pytest.raises(ValueError):
        amp.tail_matrix([("ry(0.3)", [0])])


def test_l2_probe_rejects_bad_sizes():
    """gsb_probe_l2_copy checks its arguments before touching a device: buffers of 1-64 MiB, 1-100000 passes."""
    import gsb
    for kw in (dict(mib=0), dict(mib=65), dict(mib=16, reps=0)):
        try:
            gsb.probe_l2_copy(**kw)
        except gsb.GsbError as e:
            assert e.code == 1, kw
        else:
            raise AssertionError(f"accepted {kw}")
