"""Sliced in-place plans and the twist file (drop-in for the reference's ``sliced_plans.py``:
``make_sliced_plans`` sliced_plans.py:41-86, ``gf2_solve`` :29-39, ``profile`` :26-27).

The sum being split.  With a = x_S the values of the slice vertices S,

    Z = sum_a  P(a) * sum_{x'} (-1)^{x'^T A'_< x'} prod_{u not in S} w_u(x_u) (-1)^{x_u <A[u, S], a>},
    P(a) = prod_{v in S} w_v(a_v) * (-1)^{a^T A[S, S]_< a},

where A' is A with the rows and columns of S cleared.  Every assignment a therefore runs the same plan (that of A'),
and differs only in its step matrices:
  * M_v of a slice vertex keeps its column a_v (the other is zero);
  * the sign (-1)^{x_u <A[u, S], a>} of a prefix vertex u multiplies column 1 of M_u;
  * the edges inside S give the sign (-1)^{a_i a_j A[S_i, S_j]}, carried by column 1 of the later vertex S_j.
A suffix vertex u (step >= K) cannot carry its sign: the suffix runs once, on the sum of the slices' tables at step
K.  The table at step K is indexed by logical coordinates c with functional phi(c) = sum_i c_i B_i on the suffix
variables, so the sign (-1)^{<s, x_suffix>} with s = sum_{v in S, a_v = 1} (suffix part of A[v]) is the
translation c -> c + t with sum_i t_i B_i = s.  The twist file gives t per slice, split into a kept-coordinate index
shift and a coset offset, which the executor applies while summing (``gsb_resume``).

Assignment order, file names, the K default and the text formats are the reference's, so that plans, twist file and
summary are byte-identical to what the reference writes.
"""
import json

import numpy as np

from inplace import plan_inplace, write_inplace_plan
from tableau import rank_of_ints


def _order_masks(A, order):
    """Per vertex u: bit j set when u is adjacent to order[j]."""
    A = np.asarray(A)
    cols = np.asarray(order, dtype=np.int64)
    return {u: sum(1 << int(j) for j in np.nonzero(A[u, cols] & 1)[0]) for u in range(len(A))}


def profile(A, order, ks=None):
    """{k: GF(2) rank of the cut between order[:k] and order[k:]} for k in ks (default 1..n-1)."""
    n = len(A)
    masks = _order_masks(A, order)
    out = {}
    for k in (ks or range(1, n)):
        low = (1 << k) - 1
        out[k] = rank_of_ints([masks[int(u)] & low for u in order[k:]])
    return out


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


def _popcount(x):
    return bin(x).count("1")


def _negate_col1(m, times):
    """Column 1 of a 2x2 step matrix multiplied by -1, `times` times (the complex product by -1 is applied once per
    sign factor, which fixes the signs of zero components exactly as a sequence of such products does)."""
    if not times:
        return m
    m = m.copy()
    for _ in range(times):
        m[:, 1] *= -1
    return m


def _default_K(sv, ND):
    """First step of the data-vertex suffix: just after the last ancilla (vertex >= ND); all steps when none."""
    last = max((i for i, v in enumerate(sv) if v >= ND), default=-1)
    return last + 1 if last >= 0 else len(sv)


def make_sliced_plans(A, M, order, S, out, K=None, ND=70):
    """Write one plan per assignment of the slice vertices S (``{out}_s<bits>.txt``), the twist file when a slice
    vertex has suffix neighbours, and ``{out}_slices.json``; returns dict(R, K, twist, step_vertices)."""
    A = np.asarray(A)
    N = len(A)
    S = list(S)
    s = len(S)
    Acut = A.copy()
    Acut[S, :] = 0
    Acut[:, S] = 0
    R = max(1, max(profile(Acut, order).values()))
    st = plan_inplace(Acut, order, R)
    sv = [x["v"] for x in st]
    if K is None:
        K = _default_K(sv, ND)
    prefix, suffix = set(sv[:K]), set(sv[K:])
    inS = set(S)
    for v in S:
        if v not in prefix:
            raise ValueError(f"slice vertex {v} is eliminated at or after the summation step {K}")
    # bit (s-1-i) of an assignment index is a_{S[i]}: indices 0 .. 2^s-1 enumerate the assignments in file order
    bit = [1 << (s - 1 - i) for i in range(s)]
    # per prefix vertex: the slice positions it is adjacent to; per slice vertex: the earlier slice vertices it meets
    cross = {}
    for u in prefix - inS:
        mk = sum(bit[i] for i, v in enumerate(S) if A[u, v])
        if mk:
            cross[u] = mk
    inner = [sum(bit[i] for i in range(j) if A[S[i], S[j]]) for j in range(s)]
    # per slice vertex: its suffix neighbourhood in the cut basis at step K
    trans = [0] * s
    for i, v in enumerate(S):
        sv_mask = sum(1 << int(u) for u in np.nonzero(A[v])[0] if int(u) in suffix)
        if sv_mask:
            if K >= len(st):
                raise ValueError("a slice vertex has suffix neighbours but the summation step is past the last step")
            t = gf2_solve(st[K]["B"], sv_mask)
            if t is None:
                raise ValueError(f"slice vertex {v}: its suffix neighbours are not spanned by the cut at step {K}")
            trans[i] = t
    twisted = any(trans)
    if twisted:
        keep, Tq = st[K]["keep"], st[K]["Tq"]
        keepmask = sum(1 << c for c in keep)
        q_of = {qv & ~keepmask: qv for qv in st[K]["Qall"]}   # F_2^r = span(e_keep) + Q: unique Q part
    twist = []
    for a in range(1 << s):
        Ms = list(M)
        for u, mk in cross.items():
            Ms[u] = _negate_col1(M[u], _popcount(mk & a))
        t = 0
        for i, v in enumerate(S):
            xv = 1 if a & bit[i] else 0
            mv = M[v].copy()
            mv[:, 1 - xv] = 0
            Ms[v] = _negate_col1(mv, _popcount(inner[i] & a) if xv else 0)
            if xv:
                t ^= trans[i]
        tag = "".join("1" if a & b else "0" for b in bit)
        write_inplace_plan(f"{out}_s{tag}.txt", st, R, Ms, N)
        if twisted:
            tq = q_of[t & ~keepmask]
            tk = t ^ tq
            cshift = sum(((tk >> c) & 1) << j for j, c in enumerate(keep))
            twist.append((cshift, Tq[tq]))
    if twisted:
        with open(f"{out}_twist.txt", "w") as f:
            f.write("".join(f"{c} {q}\n" for c, q in twist))
    with open(f"{out}_slices.json", "w") as f:
        json.dump({"slices": S, "R": R, "K_suffix_start": K, "twist": twisted, "step_vertices": sv}, f)
    return dict(R=R, K=K, twist=twisted, step_vertices=sv)
