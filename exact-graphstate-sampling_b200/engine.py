"""Plan and job files of the out-of-place amplitude engine, vertex slicing, and running it on the GPU.

Drop-in for the reference's ``engine.py``:
- ``write_plan`` (engine.py:5-12) and ``write_jobs`` (engine.py:38-45) write the same text formats.
- ``Sliced`` (engine.py:14-36) sums sliced vertices outside the DP.
- ``write_sampler_plan`` (engine.py:55-64) writes the two-table sampler's plan.
- ``run_dp`` (engine.py:47-53) runs the reference's dp.cpp in a gcc:14 container; here it runs this repository's
  GPU engine (libgsb ``gsb_dp_*``) in process on the same plan and jobs files.  The result is the same list of
  complex amplitudes (sum over slices of prefactor * Z).
"""
import os

import numpy as np

from plan import plan


def _parity(x):
    return bin(x).count("1") & 1


def write_plan(path, steps, m):
    maxr = max(max(s["r"], s["rn"]) for s in steps)
    with open(path, "w") as f:
        f.write(f"{m} {len(steps)} {maxr}\n")
        for s in steps:
            pm = sum(1 << p for p in s["piv"])
            f.write(f"{s['v']} {s['r']} {s['rn']} {s['rho']} {pm} {len(s['ker'])} " + " ".join(map(str, s["ker"])) + "\n")
    return maxr


class Sliced:
    """Z(w) of graph A with the vertices S summed outside the DP; the DP runs on the induced graph of the others.

    For an assignment a of the slice vertices,
        Z = sum_a  prod_{v in S} w_v(a_v) * (-1)^{a^T A[S, S]_< a} * Z_{A - S}(w^a),
    where w^a_q keeps w_q(0) and multiplies w_q(1) by (-1)^{<A[q, S], a>}.  Both signs are parities of bitmasks over
    the assignment index (bit s-1-i of the index is a_{S[i]}, so indices 0 .. 2^s-1 follow the reference's
    assignment order and its jobs file byte for byte)."""

    def __init__(self, A, order, S):
        A = np.asarray(A)
        self.A = A
        self.n = len(A)
        self.S = list(S)
        inS = set(self.S)
        self.keep = [q for q in order if q not in inS]
        self.idx = {q: i for i, q in enumerate(self.keep)}
        self.m = len(self.keep)
        self.steps = plan(np.ascontiguousarray(A[np.ix_(self.keep, self.keep)], np.uint8), list(range(self.m)))
        s = len(self.S)
        self._bit = [1 << (s - 1 - i) for i in range(s)]
        # kept vertex q: the slice positions it is adjacent to; slice position i: the later slice positions it meets
        self._cross = [sum(b for b, v in zip(self._bit, self.S) if A[q, v]) for q in self.keep]
        self._inner = [sum(self._bit[j] for j in range(i + 1, s) if A[self.S[i], self.S[j]]) for i in range(s)]

    def slices(self, w):
        """(prefactor, weights of the kept vertices) for every assignment of the sliced vertices."""
        S, bit = self.S, self._bit
        for a in range(1 << len(S)):
            pre = 1 + 0j
            ph = 0
            for i, v in enumerate(S):
                on = 1 if a & bit[i] else 0
                pre *= w[v][on]
                if on:
                    ph ^= _parity(self._inner[i] & a)
            pre *= -1 if ph else 1
            yield pre, [(w[q][0], -w[q][1] if _parity(mk & a) else w[q][1]) for q, mk in zip(self.keep, self._cross)]


def write_jobs(path, sl, ws):
    with open(path, "w") as f:
        f.write(f"{len(ws)}\n")
        for w in ws:
            sls = list(sl.slices(w))
            f.write(f"{len(sls)}\n")
            for pre, ww in sls:
                f.write("%.17g %.17g\n" % (pre.real, pre.imag))
                for a, b in ww:
                    f.write("%.17g %.17g %.17g %.17g\n" % (a.real, a.imag, b.real, b.imag))


def read_jobs(path, m):
    """Parse a jobs file for a plan of m vertices: jobs, each a list of (prefactor, [(w0, w1) per vertex])."""
    toks = open(path).read().split()
    p = 0

    def nxt():
        nonlocal p
        p += 1
        return toks[p - 1]

    jobs = []
    for _ in range(int(nxt())):
        sls = []
        for _ in range(int(nxt())):
            pre = complex(float(nxt()), float(nxt()))
            ww = []
            for _ in range(m):
                a = complex(float(nxt()), float(nxt()))
                b = complex(float(nxt()), float(nxt()))
                ww.append((a, b))
            sls.append((pre, ww))
        jobs.append(sls)
    return jobs


def run_dp(workdir, plan_file, jobs_file, threads=16, mem="8g", precision=128, device=0):
    """Amplitudes of every job of `jobs_file` under `plan_file` (paths relative to `workdir`), on the GPU.
    `threads` and `mem` (the reference's container settings) are accepted for signature compatibility."""
    import gsb
    text = open(os.path.join(workdir, plan_file)).read()
    with gsb.DpEngine(text, precision=precision, device=device) as eng:
        jobs = read_jobs(os.path.join(workdir, jobs_file), eng.m)
        return [eng.run(sls) for sls in jobs]


def write_sampler_plan(path, am):
    """Plan + per-step measurement matrices M_v (rows b, columns x) for the two-table sampler."""
    maxr = max(max(s["r"], s["rn"]) for s in am.steps)
    with open(path, "w") as f:
        f.write(f"{am.n} {len(am.steps)} {maxr}\n")
        for s in am.steps:
            pm = sum(1 << p for p in s["piv"])
            M = am.M[s["v"]]
            f.write(f"{s['v']} {s['r']} {s['rn']} {s['rho']} {pm} {len(s['ker'])} " + " ".join(map(str, s["ker"])) + " "
                    + " ".join("%.17g %.17g" % (complex(M[b, x]).real, complex(M[b, x]).imag) for b in (0, 1) for x in (0, 1)) + "\n")
    return maxr
