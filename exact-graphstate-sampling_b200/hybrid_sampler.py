"""Hybrid rejection sampling and exact scoring with the executor in process.

Drop-in for the reference's ``doped_sampler.py`` (doped_sampler.py:1-77): same argv, same output lines, same
random streams.  The reference runs its executor as a subprocess per string or proposal (:25-26, 46-47, 56, 69),
each one re-parsing the plan and allocating the arena.  Here one ``gsb.Engine`` stays loaded, unsliced proposals
go to it in batches (one C-ABI call per batch of proposals), and slice plans reuse its arena by swapping their M
matrices.

  python hybrid_sampler.py sample <plan> <step_vertices.json> <nprop> <seed> <cap> <out.txt> [--m M]
  python hybrid_sampler.py score  <plan> <step_vertices.json> <strings.txt> <out.txt> [--qiskit]
  options: --na NA (ancillas, default 468) --nd ND (data qubits, default 70) --slices s0,s1,... --K K --twist file
           --precision 64|128 (arena; default 64 like the reference's default build) --device D

Conventions (the reference's):
- Data strings are ND bits by qubit, and ancilla bits are 0.
- log2 Pr_doped(b) = log2 Pr_gadget(b, anc = 0) + NA.
- Proposals draw the first ND - m data bits uniformly, then run one hybrid pass.  That pass gives the exact marginal
  Pr(prefix, anc = 0) and an exact draw of the last m bits.
- A proposal is accepted with probability z / cap, z = 2^(ND - m) 2^NA Pr(prefix, anc = 0).
"""
import json
import math
import os
import random
import sys
import time

import gsb


class HybridSampler:
    def __init__(self, plan, step_vertices, na=468, nd=70, m=None, slices=None, K=None, twist=None, precision=64,
                 device=0):
        self.sv = json.load(open(step_vertices)) if isinstance(step_vertices, str) else list(step_vertices)
        self.ns = len(self.sv)
        self.pos = {v: i for i, v in enumerate(self.sv)}
        self.NA, self.ND = na, nd
        ms = 0
        while ms < self.ns and self.sv[self.ns - 1 - ms] < nd:
            ms += 1
        self.m_suffix = min(ms, int(m)) if m is not None else ms
        self.slices = list(slices) if slices else []
        self.KS = K
        self.twist = None
        if twist:
            self.twist = [tuple(int(x) for x in ln.split()) for ln in open(twist) if ln.strip()]
        first = self.slices[0] if self.slices else plan
        self.eng = gsb.Engine(first, precision=precision, device=device)
        self.slice_texts = [open(p).read() for p in self.slices]
        assert self.eng.ns == self.ns, "step_vertices does not match the plan"
        if not self.slices:
            # proposals force every step before the sampled suffix: those run as fused passes
            self.eng.set_hybrid_prefix(self.ns - self.m_suffix)

    def to_step_string(self, bits, free_suffix):
        s = [0] * self.ns
        for q in range(self.ND):
            s[self.pos[q]] = int(bits[q])
        if free_suffix:
            for i in range(self.ns - self.m_suffix, self.ns):
                s[i] = -1
        return s

    def sliced_eval(self, line, seed):
        """prefix on every slice plan up to K, resume on the summed dumps (with the twist): (bits, lp_full, lp_prefix,
        conditionals) as the reference's resume line prints them (doped_sampler.py:42-47)."""
        dumps, lss = [], []
        for text in self.slice_texts:
            self.eng.set_matrices_from_text(text)
            d, ls, _ = self.eng.prefix(line, self.KS)
            dumps.append(d)
            lss.append(ls)
        self.eng.set_matrices_from_text(self.slice_texts[0])
        return self.eng.resume(line, self.KS, seed, 0, dumps, lss, twist=self.twist)

    def score(self, strings_path, out_path, qiskit=False):
        lines = [ln.strip() for ln in open(strings_path) if ln.strip()]
        done = sum(1 for _ in open(out_path)) if os.path.exists(out_path) else 0
        with open(out_path, "a") as f:
            for s in lines[done:]:
                assert len(s) == self.ND and set(s) <= {"0", "1"}
                b = [int(s[self.ND - 1 - q]) for q in range(self.ND)] if qiskit else [int(c) for c in s]
                t0 = time.time()
                line = self.to_step_string(b, False)
                if self.slices:
                    lp = self.sliced_eval(line, 0)[1] + self.NA
                else:
                    lp = float(self.eng.prob([line])[0]) + self.NA
                f.write(f"{s} {lp:.9f} {time.time() - t0:.1f}\n")
                f.flush()

    def _hybrid_batches(self, props, seed):
        """Unsliced proposals evaluated BATCH at a time: one gsb_hybrid call per batch replays the hybrid graph for
        every line back to back (no host round trip between proposals).  Line i of the call draws its '?' bits from
        mt19937_64(seed * 1000003 + i), the stream the reference gives proposal i (doped_sampler.py:69).
        Yields (bits, log2 Pr, conditionals, seconds per proposal of its batch) per proposal."""
        for i0 in range(0, len(props), self.BATCH):
            lines = [self.to_step_string(p, True) for p in props[i0:i0 + self.BATCH]]
            t0 = time.time()
            bits, lpv, cond = self.eng.hybrid(lines, seed * 1000003, first_line=i0)
            dt = (time.time() - t0) / len(lines)
            for j in range(len(lines)):
                yield bits[j], float(lpv[j]), cond[j], dt

    BATCH = 64

    def sample(self, nprop, seed, cap, out_path):
        rng = random.Random(seed)
        props = [[rng.randrange(2) for _ in range(self.ND)] for _ in range(nprop)]
        u = [rng.random() for _ in range(nprop)]
        K = self.ns - self.m_suffix
        zmax, acc = 0.0, 0
        batched = None if self.slices else self._hybrid_batches(props, seed)
        with open(out_path, "a") as f:
            f.write(f"# seed {seed} cap {cap} m_suffix {self.m_suffix} K {K} nprop {nprop}\n")
            for i in range(nprop):
                t0 = time.time()
                if self.slices:
                    line = self.to_step_string(props[i], True)
                    bits, lp_full, lp_prefix, _ = self.sliced_eval(line, seed * 1000003 + i)
                    lp_full += self.NA
                    lp_prefix += self.NA
                    dt = time.time() - t0
                else:
                    bits, lp_full, cond, dt = next(batched)
                    lp_full += self.NA
                    lp_prefix = (sum(math.log2(c) for c in cond[:K]) + self.NA) if all(c > 0 for c in cond[:K]) else -math.inf
                bits_step = "".join(str(int(x)) for x in bits)
                z = 2.0 ** (lp_prefix + (self.ND - self.m_suffix))
                zmax = max(zmax, z)
                ok = u[i] < z / cap
                b = "".join(bits_step[self.pos[q]] for q in range(self.ND))
                f.write(f"{'ACC' if ok else 'rej'} {b} {lp_full:.9f} z={z:.6f} {dt:.1f}s"
                        f"{' Z_ABOVE_CAP' if z > cap else ''}\n")
                f.flush()
                acc += ok
            f.write(f"# done: {acc} accepted of {nprop}; max z {zmax:.6f}; cap {cap}\n")
        return acc, zmax

    def close(self):
        self.eng.close()


def _argval(argv, flag, default=None):
    if flag in argv:
        i = argv.index(flag)
        v = argv[i + 1]
        del argv[i:i + 2]
        return v
    return default


def main(argv):
    argv = list(argv)
    na = int(_argval(argv, "--na", 468))
    nd = int(_argval(argv, "--nd", 70))
    _argval(argv, "--threads", None)
    _argval(argv, "--bin", None)
    m = _argval(argv, "--m", None)
    slices = _argval(argv, "--slices", None)
    K = _argval(argv, "--K", None)
    twist = _argval(argv, "--twist", None)
    prec = int(_argval(argv, "--precision", 64))
    dev = int(_argval(argv, "--device", 0))
    qiskit = "--qiskit" in argv
    if qiskit:
        argv.remove("--qiskit")
    mode, plan, svj = argv[1:4]
    hs = HybridSampler(plan, svj, na=na, nd=nd, m=m, slices=slices.split(",") if slices else None,
                       K=int(K) if K else None, twist=twist, precision=prec, device=dev)
    if mode == "score":
        hs.score(argv[4], argv[5], qiskit=qiskit)
    elif mode == "sample":
        acc, zmax = hs.sample(int(argv[4]), int(argv[5]), float(argv[6]), argv[7])
        print(f"{acc} accepted of {int(argv[4])}; max z {zmax:.6f} (cap {float(argv[6])})")
    else:
        raise SystemExit("mode must be sample or score")
    hs.close()


if __name__ == "__main__":
    main(sys.argv)
