"""In-place cut-rank DP plan: the whole DP runs in one arena of 2^R complex entries (R = largest cut rank).

Drop-in for the reference's ``inplace.py`` (``plan_inplace`` inplace.py:31-100, ``sample_chain_probs``
inplace.py:102-141, ``write_inplace_plan`` inplace.py:143-159).  The plan text this module writes is the input
format of the GPU executor (and of the reference's gsamp2), so every index it contains must match the reference
bit for bit; the procedure below therefore makes exactly the reference's choices:

* Each step maps old coordinates (c, x_v) to new ones by a GF(2)-linear map with kernel K.  Q is the span of the
  old-coordinate parts of K, kept in fully reduced echelon form in insertion order; its pivot coordinates are
  dropped, the others ("keep") index the cosets c + Q, ordered by their physical address so that consecutive c
  land on nearby addresses.
* The elements (qv, x) of Q x {0,1} are grouped by their image under the map (their class modulo K), in the order
  qv enumerates Q (basis vectors doubling the list) and x = 0, 1; class tau = 0 is the class of 0.  There are m = 1
  or 2 classes, the m outputs of every coset.
* Physical addresses are a linear map T from logical coordinates to arena bits.  Kept coordinates keep their
  column; a second output goes to T(e) for the first Q basis vector e (a slot of the same coset), or, when Q = 0,
  to the lowest arena bit outside span(T) (growth).  Every coset therefore reads and overwrites only its own slots.
"""
from plan import Eliminator, adjacency_rows, step_generators


class _Rref:
    """Fully reduced echelon basis in insertion order: list of [vector, pivot bit]."""

    def __init__(self, vecs=()):
        self.rows = []
        for v in vecs:
            self.insert(v)

    def reduce(self, v):
        for b, p in self.rows:
            if (v >> p) & 1:
                v ^= b
        return v

    def insert(self, v):
        v = self.reduce(v)
        if not v:
            return False
        p = v.bit_length() - 1
        self.rows = [[b ^ v if (b >> p) & 1 else b, pb] for b, pb in self.rows]
        self.rows.append([v, p])
        return True

    def contains(self, v):
        return self.reduce(v) == 0


def _xor_cols(cols, mask):
    a = 0
    i = 0
    while mask:
        if mask & 1:
            a ^= cols[i]
        mask >>= 1
        i += 1
    return a


def _span_list(basis):
    """All elements of span(basis), enumerated by doubling (element order matters for the plan's term order)."""
    out = [0]
    for b in basis:
        out += [a ^ b for a in out]
    return out


def plan_inplace(A, order, R):
    nb = adjacency_rows(A)
    B, T = [], []
    done = 0
    steps = []
    for v in order:
        r = len(B)
        vb = 1 << v
        done |= vb
        rho = sum(1 << j for j, b in enumerate(B) if b & vb)
        gens = step_generators(B, v, nb[v], done)          # index r is x_v
        el = Eliminator()
        K = []
        for g in gens:
            new, comb = el.add(g)
            if not new:
                K.append(comb)
        low = (1 << r) - 1
        Q = _Rref(k & low for k in K if k & low)
        qbasis = [b for b, _ in Q.rows]
        qpiv = {p for _, p in Q.rows}
        keep = sorted((i for i in range(r) if i not in qpiv), key=lambda i: T[i])
        Qall = _span_list(qbasis)
        Kset = set(_span_list(K))
        reps, terms = [], []
        for qv in Qall:
            for x in (0, 1):
                u = qv | (x << r)
                tau = next((ti for ti, rep in enumerate(reps) if (u ^ rep) in Kset), None)
                if tau is None:
                    reps.append(u)
                    tau = len(reps) - 1
                terms.append((qv, x, tau))
        m = len(reps)
        assert m in (1, 2) and reps[0] == 0

        def field(u):
            return _xor_cols(gens, u)

        newB = [gens[i] for i in keep] + ([field(reps[1])] if m == 2 else [])
        if m == 2:
            if qbasis:
                g = _xor_cols(T, qbasis[0] & low)
            else:
                span_T = _Rref(T)
                g = next(1 << j for j in range(R) if not span_T.contains(1 << j))
            newT = [T[i] for i in keep] + [g]
        else:
            newT = [T[i] for i in keep]
        assert all(t < (1 << R) for t in newT) and len(_Rref(newT).rows) == len(newT), "layout not injective"
        nbasis = _Rref(newB)
        assert len(nbasis.rows) == len(newB)
        assert all(nbasis.contains(field(1 << i)) for i in range(r + 1))
        Tq = {qv: _xor_cols(T, qv) for qv in Qall}
        steps.append(dict(v=v, r=r, rn=len(newB), keep=keep, Tkeep=[T[i] for i in keep], rho=rho, terms=terms,
                          Tq=Tq, m=m, g=(newT[-1] if m == 2 else None), B=list(B), Qall=Qall))
        B, T = newB, newT
    assert not B
    return steps


def _parity(x):
    return bin(x).count("1") & 1


def inplace_plan_text(steps, R, M, n):
    """The plan text gsamp2 and the GPU executor read (reference inplace.py:143-159):
    header ``n nsteps R``; per step ``v nk m g rhoc nterms``, the nk Tkeep addresses, nterms x ``Tq x tau par``,
    then M[b][x] for b, x in (0,1)^2 as ``re im`` pairs printed with %.17g."""
    out = [f"{n} {len(steps)} {R}\n"]
    for s in steps:
        rhoc = sum(((s["rho"] >> i) & 1) << j for j, i in enumerate(s["keep"]))   # bit j of c is coordinate keep[j]
        Mv = M[s["v"]]
        head = f"{s['v']} {len(s['keep'])} {s['m']} {s['g'] or 0} {rhoc} {len(s['terms'])} "
        tk = " ".join(str(t) for t in s["Tkeep"]) + " "
        tm = " ".join(f"{s['Tq'][qv]} {x} {tau} {_parity(qv & s['rho'])}" for qv, x, tau in s["terms"]) + " "
        mm = " ".join("%.17g %.17g" % (complex(Mv[b, x]).real, complex(Mv[b, x]).imag) for b in (0, 1) for x in (0, 1))
        out.append(head + tk + tm + mm + "\n")
    return "".join(out)


def write_inplace_plan(path, steps, R, M, n):
    with open(path, "w") as f:
        f.write(inplace_plan_text(steps, R, M, n))


def sample_chain_probs(steps, R, M, bits, precision=128):
    """Exact conditionals Pr(b_k | b_1..b_{k-1}) along the forced step-order path ``bits``, evaluated on the GPU
    executor with the in-place layout (drop-in for reference inplace.py:102-141, which evaluates them in Python).
    The layout invariants the reference asserts while executing (no coset writes another coset's slots) are checked
    structurally on the plan when the executor loads it."""
    import gsb
    n = len(M)
    with gsb.Engine.from_text(inplace_plan_text(steps, R, M, n), precision=precision) as eng:
        lp, cond = eng.chain([list(bits)])
    return [float(c) for c in cond[0]]


def step_vertices(steps):
    return [s["v"] for s in steps]


def plan_width(steps):
    return max(max(s["r"], s["rn"]) for s in steps) if steps else 0


__all__ = ["plan_inplace", "sample_chain_probs", "write_inplace_plan", "inplace_plan_text", "step_vertices",
           "plan_width"]
