"""Host planning is exact integer work and must match the reference bit for bit (CPU only).

The fixtures (tests/golden/planner_cases.json) hold, for 42 circuits, what the reference's own code computes
(tableau.py, graphform.py, amp.py, plan.py, inplace.py): the graph form A, the local Cliffords U (as exact hex
floats), the out-of-place plan steps, and the in-place plan text.  This repository's modules must reproduce all of
them exactly, including the %.17g-printed M_j, which pins the floating-point matrix products too.
"""
import itertools
import json
import os

import numpy as np

from conftest import case_plan_text


def test_graph_form_and_plans_bit_exact(planner_cases):
    from circuits import tableau_of
    from graphform import graph_form
    for case in planner_cases["cases"]:
        n = case["n"]
        A, U = graph_form(tableau_of(n, case["body"]))
        assert ["".join(str(int(x)) for x in row) for row in A] == case["A"], case["name"]
        got_U = [[[float(z.real).hex(), float(z.imag).hex()] for z in u.reshape(-1)] for u in U]
        assert got_U == case["U"], case["name"]
        text, am, st, R = case_plan_text(case)
        steps = [dict(v=s["v"], r=s["r"], rn=s["rn"], rho=s["rho"], piv=s["piv"], ker=s["ker"]) for s in am.steps]
        assert steps == case["plan"], case["name"]
        assert R == case["R"]
        assert text == case["inplace_plan"], case["name"]


def test_width30_plan_regenerated(w30_dir):
    """The #151 instance (nq70.qasm + order_w30.json) through this repository's planner writes exactly the plan
    the reference's current planner writes (nq70_inplace_plan_regen.txt)."""
    from amp import Amplitudes
    from inplace import inplace_plan_text, plan_inplace
    from tableau import clifford_body
    n, T, tail = clifford_body(os.path.join(w30_dir, "nq70.qasm"))
    order = json.load(open(os.path.join(w30_dir, "order_w30.json")))
    am = Amplitudes(n, T, tail, order)
    st = plan_inplace(am.A, order, 30)
    assert inplace_plan_text(st, 30, am.M, n) == open(os.path.join(w30_dir, "nq70_inplace_plan_regen.txt")).read()


def test_shipped_width30_plan_is_an_older_layout(w30_dir):
    """The shipped plan predates the reference's physical-address ordering of kept coordinates: same step vertices
    and table sizes, different layout; both validate."""
    import gsb
    a = open(os.path.join(w30_dir, "nq70_inplace_plan.txt")).read()
    b = open(os.path.join(w30_dir, "nq70_inplace_plan_regen.txt")).read()
    assert gsb.validate_text(a) == gsb.validate_text(b) == (70, 70, 30)
    la = [ln.split() for ln in a.strip().split("\n")][1:]
    lb = [ln.split() for ln in b.strip().split("\n")][1:]
    assert [(x[0], x[1], x[2], x[5]) for x in la] == [(x[0], x[1], x[2], x[5]) for x in lb]
    assert a != b


def test_tableau_matches_dense_states():
    """Every generator stabilises C|0> with its sign (reference test_tableau.py), incl. sdg, sxdg."""
    import random
    from oracle import statevector
    from tableau import Tableau
    X = np.array([[0, 1], [1, 0]])
    Z = np.diag([1, -1])
    Y = 1j * X @ Z
    rng = random.Random(1)
    worst = 0.0
    for _ in range(80):
        n = rng.randint(2, 5)
        ops = []
        for _ in range(rng.randint(1, 40)):
            g = rng.choice(["h", "s", "sdg", "sx", "sxdg", "x", "z", "cz", "cz"])
            ops.append((g, rng.sample(range(n), 2)) if g == "cz" else (g, [rng.randrange(n)]))
        T = Tableau(n)
        for g, qs in ops:
            T.apply(g, qs)
        psi = statevector.dense_state(n, ops)
        xs, zs, r = T.xs, T.zs, T.r
        for i in range(n):
            P = np.array([[1]])
            for q in range(n):
                P = np.kron(P, {(0, 0): np.eye(2), (1, 0): X, (0, 1): Z, (1, 1): Y}[(int(xs[i, q]), int(zs[i, q]))])
            worst = max(worst, np.linalg.norm((-1) ** int(r[i]) * P @ psi - psi))
    assert worst < 1e-12


def test_amplitudes_vs_statevector(planner_cases):
    """<b|psi> = 2^{-n/2} sum_x prod_j M_j[b_j, x_j] (-1)^{x^T A x} against dense states (reference test_amp.py),
    for every string of the small cases; negative control U instead of U^dag."""
    from amp import Amplitudes
    from circuits import tableau_of
    from graphform import graph_form
    from oracle import statevector
    worst, ctrl = 0.0, 0.0
    for case in planner_cases["cases"]:
        n = case["n"]
        if n > 8:
            continue
        T = tableau_of(n, case["body"])
        am = Amplitudes(n, T, [tuple(x) for x in case["tail"]], case["order"])
        ops = [tuple(x) for x in case["body"]] + [tuple(x) for x in case["tail"]]
        psi2 = statevector.probabilities(n, ops)
        xs = np.array(list(itertools.product((0, 1), repeat=n)))
        ph = (-1.0) ** (np.einsum("ki,ij,kj->k", xs, np.triu(am.A, 1), xs) % 2)
        _, U = graph_form(T)
        for idx, b in enumerate(itertools.product((0, 1), repeat=n)):
            w = np.prod([am.M[q][b[q], xs[:, q]] for q in range(n)], axis=0)
            amp = (w * ph).sum() / 2 ** (n / 2)
            worst = max(worst, abs(abs(amp) ** 2 - psi2[idx]))
            if idx < 4:
                Mb = [am.W[q] @ U[q] for q in range(n)]
                wb = np.prod([Mb[q][b[q], xs[:, q]] for q in range(n)], axis=0)
                ctrl = max(ctrl, abs(abs((wb * ph).sum()) ** 2 / 2 ** n - psi2[idx]))
    assert worst < 1e-12 and ctrl > 1e-3


def test_native_cut_profile_and_order_search(planner_cases):
    import gsb
    from plan import plan
    for case in planner_cases["cases"]:
        A = np.array([[int(ch) for ch in row] for row in case["A"]], np.uint8)
        prof = gsb.cut_profile(A, case["order"])
        steps = plan(A, case["order"])
        assert prof == [s["rn"] for s in steps[:-1]]
    c1 = [c for c in planner_cases["cases"] if c["name"] == "config1_n20"][0]
    A = np.array([[int(ch) for ch in row] for row in c1["A"]], np.uint8)
    order, w = gsb.order_search(A, seed=11, ngreedy=4, iters=20000)
    assert sorted(order) == list(range(20)) and w == max(gsb.cut_profile(A, order)) and w <= 10


def _am_of(case):
    from amp import Amplitudes
    from circuits import tableau_of
    return Amplitudes(case["n"], tableau_of(case["n"], case["body"]), [tuple(t) for t in case["tail"]], case["order"])


def test_engine_plan_and_jobs_text(planner_cases, tmp_path):
    """engine.write_plan / Sliced / write_jobs write the reference's text byte for byte (engine.py:5-45)."""
    import json
    from conftest import GOLDEN
    from engine import Sliced, write_jobs, write_plan
    extras = json.load(open(os.path.join(GOLDEN, "extras_cases.json")))
    cases = {c["name"]: c for c in planner_cases["cases"]}
    for d in extras["dp"]:
        am = _am_of(cases[d["name"]])
        sl = Sliced(am.A, cases[d["name"]]["order"], d["S"])
        write_plan(str(tmp_path / "p.txt"), sl.steps, sl.m)
        write_jobs(str(tmp_path / "j.txt"), sl, [am.weights(b) for b in d["bits"]])
        assert (tmp_path / "p.txt").read_text() == d["plan"]
        assert (tmp_path / "j.txt").read_text() == d["jobs"]


def test_sliced_plans_and_twist(planner_cases, tmp_path):
    """make_sliced_plans writes the reference's slice plans, twist file and summary (sliced_plans.py:41-86)."""
    import json
    from conftest import GOLDEN
    from sliced_plans import make_sliced_plans
    extras = json.load(open(os.path.join(GOLDEN, "extras_cases.json")))
    cases = {c["name"]: c for c in planner_cases["cases"]}
    assert extras["sliced"]
    for d in extras["sliced"]:
        c = cases[d["name"]]
        am = _am_of(c)
        out = str(tmp_path / "sp")
        info = make_sliced_plans(am.A, [m.copy() for m in am.M], c["order"], d["S"], out, K=d["K"], ND=c["n"])
        assert info == d["info"]
        for tag, text in d["plans"].items():
            assert open(f"{out}_s{tag}.txt").read() == text
        assert open(f"{out}_twist.txt").read() == d["twist"]
        assert open(f"{out}_slices.json").read() == d["slices_json"]
