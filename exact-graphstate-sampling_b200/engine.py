"""Plan and job files of the out-of-place amplitude engine, vertex slicing, and running it on the GPU.

Drop-in for the reference's ``engine.py``:
- ``write_plan`` (engine.py:5-12) and ``write_jobs`` (engine.py:38-45) write the same text formats.
- ``Sliced`` (engine.py:14-36) sums sliced vertices outside the DP.
- ``write_sampler_plan`` (engine.py:55-64) writes the two-table sampler's plan.
- ``run_dp`` (engine.py:47-53) runs the reference's dp.cpp in a gcc:14 container; here it runs this repository's
  GPU engine (libgsb ``gsb_dp_*``) in process on the same plan and jobs files.  The result is the same list of
  complex amplitudes (sum over slices of prefactor * Z).
"""
import itertools
import os

import numpy as np

from plan import plan


def write_plan(path, steps, m):
    maxr = max(max(s["r"], s["rn"]) for s in steps)
    with open(path, "w") as f:
        f.write(f"{m} {len(steps)} {maxr}\n")
        for s in steps:
            pm = sum(1 << p for p in s["piv"])
            f.write(f"{s['v']} {s['r']} {s['rn']} {s['rho']} {pm} {len(s['ker'])} " + " ".join(map(str, s["ker"])) + "\n")
    return maxr


class Sliced:
    """Z(w) for graph A with the vertices in S summed outside the DP (graph A - S inside)."""

    def __init__(self, A, order, S):
        n = len(A)
        self.S = list(S)
        Sset = set(S)
        self.keep = [q for q in order if q not in Sset]
        self.idx = {q: i for i, q in enumerate(self.keep)}
        m = len(self.keep)
        Ak = np.zeros((m, m), np.uint8)
        for i, p in enumerate(self.keep):
            for j, q in enumerate(self.keep):
                Ak[i, j] = A[p, q]
        self.A = A
        self.m = m
        self.n = n
        self.steps = plan(Ak, list(range(m)))

    def slices(self, w):
        """(prefactor, weights of the kept vertices) for every assignment of the sliced vertices."""
        A, S = self.A, self.S
        for xs in itertools.product((0, 1), repeat=len(S)):
            pre = 1 + 0j
            ph = 0
            for a, (v, xv) in enumerate(zip(S, xs)):
                pre *= w[v][xv]
                for v2, x2 in list(zip(S, xs))[a + 1:]:
                    ph ^= int(A[v, v2]) & xv & x2
            pre *= (-1) ** ph
            ww = []
            for q in self.keep:
                f = sum(int(A[q, v]) & xv for v, xv in zip(S, xs)) & 1
                ww.append((w[q][0], -w[q][1] if f else w[q][1]))
            yield pre, ww


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
