"""The reference executor's command line, `gsb2` / `gsb2_c128`, on the GPU: every mode gives the compiled reference
executor's recorded output lines (gsamp2.cpp:149-225) and its exit codes.

Process-based callers switch executors by path (doped_sampler.py --bin, doped_sampler.py:28), so this is the
reference's own plug-in seam.  Lines are compared field by field: bit strings and indices exactly, log2 Pr and
conditionals within the form's tolerance (complex128: 1e-9; complex64: 1e-5 in log2 Pr, 1e-6 in conditionals, as the
C-ABI parity tests hold them), printf formats by the number of digits after the point.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, PKG

pytestmark = pytest.mark.gpu

TOL = {128: (1e-9, 1e-9), 64: (1e-5, 1e-6)}     # (log2 Pr, conditionals)


def gsb2(prec, args, cwd):
    exe = os.path.join(PKG, "gsb2_c128" if prec == 128 else "gsb2")
    return subprocess.run([exe] + [str(a) for a in args], cwd=cwd, capture_output=True, text=True, timeout=600)


def _digits(tok):
    return len(tok.split(".")[1]) if "." in tok else -1


def same_line(got, ref, prec, kinds):
    """kinds: per field, 'x' exact, 'p' log2 Pr, 'c' conditional, 'l' logscale (%.6f)."""
    g, r = got.split(), ref.split()
    assert len(g) == len(r), (got, ref)
    tp, tc = TOL[prec]
    for i, (a, b) in enumerate(zip(g, r)):
        k = kinds[i] if i < len(kinds) else kinds[-1]
        if k == "x":
            assert a == b, (i, got, ref)
            continue
        assert _digits(a) == _digits(b), (i, a, b)
        if a in ("-inf", "inf", "nan") or b in ("-inf", "inf", "nan"):
            assert a == b, (i, got, ref)
            continue
        tol = {"p": tp, "c": tc, "l": 1e-5}[k]
        assert abs(float(a) - float(b)) <= tol, (i, a, b, tol)


def _plans():
    return {c["name"]: c["inplace_plan"] for c in json.load(open(os.path.join(GOLDEN, "planner_cases.json")))["cases"]}


@pytest.mark.parametrize("prec", [128, 64])
def test_cli_every_mode_matches_reference_lines(executor_cases, prec, tmp_path):
    plans = _plans()
    for ec in executor_cases:
        d = tmp_path / ec["name"]
        d.mkdir()
        (d / "p.txt").write_text(plans[ec["name"]])
        (d / "s.txt").write_text("\n".join(ec["strings"]) + "\n")
        (d / "h.txt").write_text("\n".join(ec["hybrid_lines"]) + "\n")
        (d / "pre.txt").write_text("\n".join(ec["prefix_lines"]) + "\n")
        K = int(ec["K"])
        runs = [
            (["p.txt", "prob", "s.txt"], f"prob{prec}", "p"),
            (["p.txt", "chain", "s.txt"], f"chain{prec}", "pc"),
            (["p.txt", "sample", 40, 1000], f"sample{prec}", "xpx"),
            (["p.txt", "sample2", 12, 5], f"sample2_{prec}", "xpx"),
            (["p.txt", "hybrid", "h.txt", 9], f"hybrid{prec}", "xpc"),
            (["p.txt", "prefix", "pre.txt", K, "d"], f"prefix{prec}", "xpl"),
            (["p.txt", "resume", "pre.txt", K, 3, "d"], f"resume{prec}", "xppc"),
        ]
        for args, key, kinds in runs:
            r = gsb2(prec, args, d)
            assert r.returncode == 0, (ec["name"], args, r.stderr)
            got = [ln for ln in r.stdout.split("\n") if ln.strip()]
            ref = [ln for ln in ec[key] if ln.strip()]
            assert len(got) == len(ref), (ec["name"], key)
            for a, b in zip(got, ref):
                same_line(a, b, prec, kinds)


def test_cli_exit_codes(executor_cases, tmp_path):
    """The reference's exit codes: 1 usage, 2-6 plan parse, 8 '?' before K, 9 missing dump, 10 bad dump,
    12 missing twist file, 13 bad twist line."""
    plans = _plans()
    ec = executor_cases[0]
    d = tmp_path
    (d / "p.txt").write_text(plans[ec["name"]])
    (d / "s.txt").write_text("\n".join(ec["strings"]) + "\n")
    ns = len(ec["strings"][0])
    K = int(ec["K"])
    assert gsb2(64, ["p.txt", "prob"], d).returncode == 1
    (d / "bad.txt").write_text("garbage")
    assert gsb2(64, ["bad.txt", "prob", "s.txt"], d).returncode == 2
    lines = plans[ec["name"]].split("\n")
    (d / "trunc.txt").write_text(lines[0] + "\n" + " ".join(lines[1].split()[:3]) + "\n")
    assert gsb2(64, ["trunc.txt", "prob", "s.txt"], d).returncode == 3
    (d / "q.txt").write_text("?" * ns + "\n")
    assert gsb2(64, ["p.txt", "prefix", "q.txt", K, "d"], d).returncode == 8
    (d / "pre.txt").write_text("0" * K + "?" * (ns - K) + "\n")
    assert gsb2(64, ["p.txt", "resume", "pre.txt", K, 3, "nodump"], d).returncode == 9
    assert gsb2(64, ["p.txt", "prefix", "pre.txt", K, "d"], d).returncode == 0
    raw = (d / "d_0.bin").read_bytes()
    (d / "e_0.bin").write_bytes(raw[:len(raw) - 8])
    assert gsb2(64, ["p.txt", "resume", "pre.txt", K, 3, "e"], d).returncode == 10
    assert gsb2(64, ["p.txt", "resume", "pre.txt", K, 3, "d", "--twist", "none.txt"], d).returncode == 12
    (d / "tw.txt").write_text("x y\n")
    assert gsb2(64, ["p.txt", "resume", "pre.txt", K, 3, "d", "--twist", "tw.txt"], d).returncode == 13
    # and the same run without the broken inputs succeeds
    r = gsb2(64, ["p.txt", "resume", "pre.txt", K, 3, "d"], d)
    assert r.returncode == 0 and len(r.stdout.split()) == 3 + ns - K


def test_cli_replays_the_reference_drivers_executor_calls(tmp_path):
    """Every executor call the reference's hybrid driver (doped_sampler.py, unsliced and sliced with a twist file;
    sample and score modes) made with the compiled reference executor as --bin, replayed in order against gsb2:
    the same stdout, field by field, and the same exit status.  The calls were recorded with their inputs by
    tests/golden/record_driver_calls.py, since the driver itself is not part of this repository."""
    rec = json.load(open(os.path.join(GOLDEN, "driver_calls.json")))
    plans = _plans()
    assert rec["runs"]
    for run in rec["runs"]:
        d = tmp_path / run["name"]
        d.mkdir()
        for fname, text in run["files"].items():
            (d / fname).write_text(plans[text[len("@plan:"):]] if text.startswith("@plan:") else text)
        for call in run["calls"]:
            for fname, text in call["inputs"].items():
                (d / fname).write_text(text)
            args = call["argv"][1:]
            r = gsb2(64, args, d)
            assert r.returncode == call["rc"], (run["name"], args, r.stderr)
            got = [ln for ln in r.stdout.split("\n") if ln.strip()]
            ref = [ln for ln in call["stdout"].split("\n") if ln.strip()]
            assert len(got) == len(ref), (run["name"], args)
            kinds = {"prob": "p", "hybrid": "xpc", "prefix": "xpl", "resume": "xppc"}[args[1]]
            for a, b in zip(got, ref):
                same_line(a, b, 64, kinds)
