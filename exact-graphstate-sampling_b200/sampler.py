"""Exact qubit-by-qubit sampler: the reference's ``sampler_ref`` call signatures, evaluated on the GPU.

Drop-in for ``sampler_ref.py``: ``extend`` (sampler_ref.py:8-23), ``conditionals`` (:25-33), ``chain_distribution``
(:35-46) and ``sample`` (:48-55).  Measuring the first t qubits of the DP order leaves the prefix vector P_t and
Pr(b_1..b_t) = 2^{-t} sum_c |P_t[c]|^2, so exact chain-rule sampling needs no right environment.

* ``extend`` runs one out-of-place DP step on the GPU (libgsb ``gsb_dp_extend``).
* The others run the in-place executor on the plan of ``am`` (``plan_inplace(am.A, am.order, width)``, complex128),
  built once per ``Amplitudes`` object:
  - conditionals use prefix probabilities (``prefix`` mode without the dump);
  - the full distribution uses 'chain' mode over every string;
  - samples use the chain-rule draw with ``rng.random()`` called once per step in step order, as the reference
    draws.
"""
import itertools

import numpy as np

import gsb
from inplace import inplace_plan_text, plan_inplace, plan_width


def extend(old, st, wv):
    """One DP step with weights wv = (w(0), w(1)) for the processed vertex (complex128 table in, table out)."""
    return gsb.dp_extend(np.asarray(old, np.complex128), st["r"], st["rn"], st["rho"], st["piv"], st["ker"], wv)


def _engine(am, precision=128):
    key = f"_gsb_engine_{precision}"
    eng = getattr(am, key, None)
    if eng is None:
        R = max(1, plan_width(am.steps))
        st = plan_inplace(am.A, am.order, R)
        eng = gsb.Engine.from_text(inplace_plan_text(st, R, am.M, am.n), precision=precision)
        setattr(am, key, eng)
    return eng


def conditionals(am, prefix_bits):
    """(Pr(b | prefix) for b = 0, 1 ; the two marginals Pr(prefix, b)) at step len(prefix_bits)."""
    eng = _engine(am)
    t = len(prefix_bits)
    nrm = np.zeros(2)
    for b in (0, 1):
        line = [int(x) for x in prefix_bits] + [b] + [0] * (eng.ns - t - 1)
        _, _, lp = eng.prefix(line, t + 1, want_dump=False)
        nrm[b] = 2.0 ** lp
    return nrm / nrm.sum(), nrm


def chain_distribution(am):
    """Exact distribution implied by the sampler (product of its conditionals) for every string: {bits: p}."""
    eng = _engine(am)
    ns = eng.ns
    strings = np.array(list(itertools.product((0, 1), repeat=ns)), np.int8).reshape(-1, ns)
    lp, _ = eng.chain(strings)
    out = {}
    for row, l in zip(strings, lp):
        p = 2.0 ** l if np.isfinite(l) else 0.0
        if p > 0:
            b = [0] * am.n
            for st, bv in zip(am.steps, row):
                b[st["v"]] = int(bv)
            out[tuple(b)] = p
    return out


def sample(am, rng):
    """One exact sample (bits by qubit); draws rng.random() once per step in step order."""
    eng = _engine(am)
    u = np.array([[rng.random() for _ in range(eng.ns)]])
    bits, _ = eng.sample_uniform(u)
    b = [0] * am.n
    for st, bv in zip(am.steps, bits[0]):
        b[st["v"]] = int(bv)
    return b
