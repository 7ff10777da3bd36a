"""Sliced in-place plans and the twist file (drop-in for the reference's ``sliced_plans.py``).

``make_sliced_plans`` (sliced_plans.py:41-86), ``gf2_solve`` (:29-39) and ``profile`` (:26-27).

Slicing vertex v fixes x_v: the Ising sum splits over the values of x_v, each a sum on the graph with v's edges
removed.  The weight w_v(x_v) is kept, and the phases (-1)^{x_v x_u} fold into M_u[:, 1] for every prefix neighbour
u.  All 2^{|S|} slice assignments share one graph and therefore one plan structure; only their M differ, so their
dumped tables add up (prefix / resume).  A neighbour in the suffix (steps >= K) cannot carry the folded phase,
because the suffix runs once on the summed table.  Its phase is a translation of the table at step K instead: the
twist file gives, per slice, the shift of the kept-coordinate index and of the coset offset, which the executor
applies when summing (``gsb_resume``).

The plan texts and the twist file must equal the reference's, so the choices below are the reference's:
- slice vertices are cut from A;
- the width is the largest cut rank;
- K defaults to the first step of the pure-data suffix;
- the phase folding follows slice order;
- an edge between two slice vertices is counted once, on the later vertex.
"""
import itertools
import json

import numpy as np

from inplace import plan_inplace, write_inplace_plan
from tableau import gf2_rank


def profile(A, order, ks=None):
    n = len(A)
    ks = ks or range(1, n)
    return {k: gf2_rank(A[np.ix_(order[k:], order[:k])]) for k in ks}


def gf2_solve(B, s):
    """a with XOR_i a_i B_i = s (Python ints as bit vectors), or None."""
    s = int(s)
    piv = {}                                  # leading bit -> (vector, combination mask)
    for i, b in enumerate(B):
        v, comb = int(b), 1 << i
        for lead in sorted(piv, reverse=True):
            if (v >> lead) & 1:
                v ^= piv[lead][0]
                comb ^= piv[lead][1]
        if v:
            piv[v.bit_length() - 1] = (v, comb)
    comb = 0
    for lead in sorted(piv, reverse=True):
        if (s >> lead) & 1:
            s ^= piv[lead][0]
            comb ^= piv[lead][1]
    return comb if s == 0 else None


def make_sliced_plans(A, M, order, S, out, K=None, ND=70):
    """Write the plans of every assignment of the slice vertices S; returns dict(R, K, twist, step_vertices)."""
    N = len(A)
    A2 = A.copy()
    for v in S:
        A2[v, :] = 0
        A2[:, v] = 0
    R = max(1, max(profile(A2, order).values()))
    st = plan_inplace(A2, order, R)
    sv = [s["v"] for s in st]
    if K is None:
        K = next(i for i in range(len(sv)) if all(v < ND for v in sv[i:]))
        if K == 0:
            K = len(sv)
    pre = set(sv[:K])
    suf = set(sv[K:])
    for v in S:
        assert v in pre, f"slice vertex {v} lies in the suffix"
    avec = {}
    B = keep = Tq = Qall = None
    if K < len(st):
        B, keep, Tq, Qall = st[K]["B"], st[K]["keep"], st[K]["Tq"], st[K]["Qall"]
    for v in S:
        s_v = sum(1 << int(u) for u in np.nonzero(A[v])[0] if u in suf)
        if s_v:
            assert K < len(st), "suffix neighbours but K is past the end"
            a = gf2_solve(B, s_v)
            assert a is not None, f"slice vertex {v}: suffix neighbourhood not in the span of the cut at step {K}"
            avec[v] = a
    Sset = set(S)
    twist = []
    for bits in itertools.product([0, 1], repeat=len(S)):
        Ms = [m.copy() for m in M]
        a = 0
        for v, xv in zip(S, bits):
            Ms[v][:, 1 - xv] = 0
            if xv:
                for u in np.nonzero(A[v])[0]:
                    if u in pre and u not in Sset:
                        Ms[u][:, 1] *= -1
                a ^= avec.get(v, 0)
        for i in range(len(S)):
            for j in range(i + 1, len(S)):
                if A[S[i], S[j]] and bits[i] and bits[j]:
                    Ms[S[j]][:, 1] *= -1
        tag = "".join(map(str, bits))
        write_inplace_plan(f"{out}_s{tag}.txt", st, R, Ms, N)
        if avec:
            keepmask = sum(1 << i for i in keep)
            aq = next(qv for qv in Qall if (a ^ qv) & ~keepmask == 0)
            ak = a ^ aq
            cshift = sum(((ak >> keep[j]) & 1) << j for j in range(len(keep)))
            twist.append((cshift, Tq[aq]))
    if avec:
        with open(f"{out}_twist.txt", "w") as f:
            for cshift, tqshift in twist:
                f.write(f"{cshift} {tqshift}\n")
    json.dump({"slices": S, "R": R, "K_suffix_start": K, "twist": bool(avec), "step_vertices": sv},
              open(f"{out}_slices.json", "w"))
    return dict(R=R, K=K, twist=bool(avec), step_vertices=sv)
