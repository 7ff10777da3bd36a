"""Benchmark workloads as plans: seeded circuit -> graph form -> order -> in-place plan text.

``matching_n70_w30()`` is the headline instance: n = 70, 70 layers of CZ on seeded random perfect matchings with
seeded random single-qubit Cliffords (seed 2), a Haar-random U3 per qubit, and the order the native search finds
with seed 12, whose width is 30 (arena 2^30: 8.6 GB complex64, 17.2 GB complex128).
"""
import numpy as np

import circuits
import gsb
from amp import Amplitudes
from inplace import inplace_plan_text, plan_inplace, plan_width


def build(n, body, tail, order):
    am = Amplitudes(n, circuits.tableau_of(n, body), tail, order)
    R = max(1, plan_width(am.steps))
    st = plan_inplace(am.A, order, R)
    return inplace_plan_text(st, R, am.M, n), st, R


def matching_instance(n=70, depth=70, seed=2, order_seed=12, iters=60000):
    n, body, tail = circuits.matching_circuit(n, depth, seed=seed)
    from graphform import graph_form
    A, _ = graph_form(circuits.tableau_of(n, body))
    order, w = gsb.order_search(A, seed=order_seed, ngreedy=4, iters=iters)
    text, st, R = build(n, body, tail, order)
    return dict(name=f"matching_n{n}_d{depth}_s{seed}", n=n, body=body, tail=tail, order=order, width=R, plan=text,
                steps=st)


def rotation_instance(n, depth=None, seed=0, order_seed=12, iters=60000):
    """The matching construction with its U3 layer as parameters (the differentiation workload).

    The plan is built from the Clifford body alone, so its matrices are M0_j = U_j^dag (the graph form's local
    Cliffords), and the layer's Haar angles theta0 [n, 3] are returned beside it: the step matrices of the full
    circuit are U3(theta_v) M0_v (adjoint.step_matrices)."""
    n, body, tail = circuits.matching_circuit(n, depth, seed=seed)
    from graphform import graph_form
    A, _ = graph_form(circuits.tableau_of(n, body))
    order, w = gsb.order_search(A, seed=order_seed, ngreedy=4, iters=iters)
    am = Amplitudes(n, circuits.tableau_of(n, body), [], order)
    R = max(1, plan_width(am.steps))
    st = plan_inplace(am.A, order, R)
    theta0 = np.array([[float(x) for x in name[3:-1].split(",")] for name, _ in tail])
    return dict(name=f"rotations_n{n}_d{n if depth is None else depth}_s{seed}", n=n, body=body, tail=tail,
                order=order, width=R, plan=inplace_plan_text(st, R, am.M, n), steps=st, M0=np.array(am.M),
                theta0=theta0, step_vertices=[int(x["v"]) for x in st])


def qubit_order_instance(n, depth, seed):
    """The matching construction with the qubits eliminated in index order (no order search): widths near n / 2."""
    n, body, tail = circuits.matching_circuit(n, depth, seed=seed)
    order = list(range(n))
    text, st, R = build(n, body, tail, order)
    return dict(name=f"matching_n{n}_d{depth}_s{seed}_qubit_order", n=n, body=body, tail=tail, order=order, width=R,
                plan=text, steps=st)


def batch_workload(count=512, seed=0, nmin=16, nmax=40, npre=16, nsuf=4, iters=5000, order="qubit"):
    """The batched workload: `count` matching instances with n uniform in [nmin, nmax] (instance i: circuit seed
    seed * 100003 + i), and per instance npre random prefixes over its first floor(ns/2) steps, each with nsuf random
    suffixes.  order "qubit" eliminates the qubits in index order (widths 7-20 for n in [16, 40], the widths the
    batched configuration states); "search" uses the native order search (seed 12, `iters` moves: widths 4-17).
    Returns dict(instances, K, prefixes, suffixes)."""
    rng = np.random.default_rng(seed)
    ns_list = rng.integers(nmin, nmax + 1, size=count)
    inst, K, pre, suf = [], [], [], []
    for i, n in enumerate(ns_list):
        if order == "qubit":
            w = qubit_order_instance(int(n), int(n), seed * 100003 + i)
        else:
            w = matching_instance(int(n), int(n), seed * 100003 + i, 12, iters)
        ns = len(w["steps"])
        k = ns // 2
        inst.append(w)
        K.append(k)
        pre.append(rng.integers(0, 2, size=(npre, k), dtype=np.int8))
        suf.append(rng.integers(0, 2, size=(npre, nsuf, ns - k), dtype=np.int8))
    return dict(instances=inst, K=K, prefixes=pre, suffixes=suf)


def wide34_instance():
    """The largest single-GPU width: n = 80, depth 80, circuit seed 6, order from the native search (seed 12, 8 greedy
    starts, 60000 moves) of width 34: a 2^34-entry arena, 137 GB complex64."""
    n, body, tail = circuits.matching_circuit(80, 80, seed=6)
    from graphform import graph_form
    A, _ = graph_form(circuits.tableau_of(n, body))
    order, w = gsb.order_search(A, seed=12, ngreedy=8, iters=60000)
    text, st, R = build(n, body, tail, order)
    return dict(name="matching_n80_d80_s6_w34", n=n, body=body, tail=tail, order=order, width=R, plan=text, steps=st)


WIDE34_SLICES = (4, 59, 18, 60, 67, 39, 41, 10, 2, 26)


def wide34_slices(w, S=WIDE34_SLICES, order_seed=5, iters=60000):
    """The width-34 instance's complex128 cross-check: a second order for the graph with the slice vertices S cut out
    (native search, seed 5), and the reference-format slice plans of make_sliced_plans on it, one per assignment of
    S.  The default S, ten vertices picked greedily (each the vertex whose removal lowers the widest cuts of the
    current order most), gives width 30: 1,024 slices, each a 2^30-entry complex128 arena (17.2 GB).  Every slice
    vertex and all of their neighbours are eliminated by the last step, so the slices' final tables add up with no
    twist."""
    import os
    import tempfile
    from graphform import graph_form
    from sliced_plans import make_sliced_plans
    n = w["n"]
    T = circuits.tableau_of(n, w["body"])
    A, _ = graph_form(T)
    A = np.array(A, np.uint8)
    A2 = A.copy()
    for v in S:
        A2[v, :] = 0
        A2[:, v] = 0
    order2, width2 = gsb.order_search(A2, seed=order_seed, ngreedy=4, iters=iters)
    am = Amplitudes(n, T, w["tail"], order2)
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "sl")
        info = make_sliced_plans(A, [m.copy() for m in am.M], list(order2), list(S), out, ND=n)
        plans = [open(f"{out}_s{''.join(map(str, bits))}.txt").read()
                 for bits in np.ndindex(*([2] * len(S)))]
    return dict(S=list(S), order=list(order2), width=info["R"], K=info["K"], twist=info["twist"], plans=plans,
                step_vertices=info["step_vertices"])


def matching_n70_w30():
    return matching_instance(70, 70, 2, 12, 60000)


def graph_state_instance(n=20, p=0.5, seed=1, order_seed=11, iters=20000):
    n, body, tail = circuits.graph_state_circuit(n, p, seed=seed)
    from graphform import graph_form
    A, _ = graph_form(circuits.tableau_of(n, body))
    order, w = gsb.order_search(A, seed=order_seed, ngreedy=4, iters=iters)
    text, st, R = build(n, body, tail, order)
    return dict(name=f"gnp_n{n}_s{seed}", n=n, body=body, tail=tail, order=order, width=R, plan=text, steps=st)


def twin_graph_instance(h=46, ntw=14, seed=10, p=0.5, order_seed=11, iters=8000):
    """Graph state of a G(h, p) graph plus ntw false twins (a copy of a vertex's neighbourhood), then a seeded U3 per
    qubit.  Measuring a twin after its original can leave the step with one output class (m = 1): the defaults give
    such a step at cut rank 14 (k = 35, width 19), wide enough for the fused passes' generic dataflow path."""
    rng = np.random.default_rng(seed)
    n = h + ntw
    E = {(i, j) for i in range(h) for j in range(i + 1, h) if rng.random() < p}
    for t, v in enumerate(rng.choice(h, ntw, replace=False)):
        w = h + t
        for (a, b) in list(E):
            if a == v and b < h:
                E.add((min(b, w), max(b, w)))
            if b == v and a < h:
                E.add((min(a, w), max(a, w)))
    body = [("h", [q]) for q in range(n)] + [("cz", [a, b]) for (a, b) in sorted(E)]
    tail = [circuits.u3_op(q, *(float(x) for x in rng.uniform(0, 2 * np.pi, 3))) for q in range(n)]
    from graphform import graph_form
    A, _ = graph_form(circuits.tableau_of(n, body))
    order, w = gsb.order_search(A, seed=order_seed, ngreedy=4, iters=iters)
    text, st, R = build(n, body, tail, order)
    return dict(name=f"twins_h{h}_t{ntw}_s{seed}", n=n, body=body, tail=tail, order=order, width=R, plan=text,
                steps=st)


def pass_bytes(steps, esize, passes="chain"):
    """Algorithmic bytes of one string: a write pass moves E (2^{r_k} + 2^{r_{k+1}}), a norm pass E 2^{r_k}
    (r_{k+1} = nk + log2 m).  passes: 'chain' (write only) or 'sample' (norm + write per step)."""
    tot = 0
    per = []
    for s in steps:
        r, rn = s["r"], s["rn"]
        w = esize * ((1 << r) + (1 << rn))
        nrm = esize * (1 << r) if passes == "sample" else 0
        per.append((w, nrm))
        tot += w + nrm
    return tot, per


def random_strings(ns, count, seed):
    return np.random.default_rng(seed).integers(0, 2, size=(count, ns), dtype=np.int8)
