"""Out-of-place plan of the cut-rank dynamic program for  Z(w) = sum_x prod_j w_j(x_j) (-1)^{sum_{i<j} A_ij x_i x_j}.

Drop-in for the reference's ``plan.py`` (``plan`` plan.py:12-35); the method is linear rank-width elimination
(Van den Nest, Duer, Vidal, Briegel, PRA 75, 012337 (2007)).

After the vertices of a prefix are summed out, they act on the remaining vertices only through the field
s = A[F, P] x_P, an element of an r-dimensional GF(2) space (r = cut rank).  The DP table is indexed by
coordinates c in a basis B of that space (vectors over the vertices, as Python ints).  Processing vertex v maps
(c, x_v) -> c' linearly (the map Lambda); the step is described by
    rho  : bit j set when basis vector j touches v (the sign (-1)^{x_v <rho, c>}),
    piv  : indices into the generators [B_0 & ~v, ..., B_{r-1} & ~v, N(v) \\ done] that form the new basis,
    ker  : a basis of ker Lambda, as combination masks over those generators.
The kernel basis is produced by one fixed elimination order (each generator reduced against the pivots found so
far, highest leading bit first), which is what makes the ``ker`` lists identical to the reference's.
"""


def adjacency_rows(A):
    n = len(A)
    return [sum(int(A[i][j]) << j for j in range(n)) for i in range(n)]


class Eliminator:
    """Incremental GF(2) elimination of a sequence of generators.

    ``add(vec)`` reduces ``vec`` against the pivots found so far (by decreasing leading bit) and returns
    ``(True, None)`` when it is independent (a new pivot) or ``(False, comb)`` with ``comb`` the combination mask
    over the generators added so far (bit i = generator i) that sums to zero."""

    def __init__(self):
        self.piv = {}                          # leading bit -> (reduced vector, combination mask)
        self.count = 0

    def add(self, vec):
        comb = 1 << self.count
        self.count += 1
        t = vec
        for lead in sorted(self.piv, reverse=True):
            if (t >> lead) & 1:
                bv, bc = self.piv[lead]
                t ^= bv
                comb ^= bc
        if t:
            self.piv[t.bit_length() - 1] = (t, comb)
            return True, None
        return False, comb


def step_generators(B, v, nbv, done):
    """Generators of step v: the old basis with v removed, then v's unprocessed neighbourhood (index r = x_v)."""
    vb = 1 << v
    return [b & ~vb for b in B] + [nbv & ~done]


def plan(A, order):
    nb = adjacency_rows(A)
    B = []
    done = 0
    steps = []
    for v in order:
        r = len(B)
        vb = 1 << v
        rho = sum(1 << j for j, b in enumerate(B) if b & vb)
        done |= vb
        gens = step_generators(B, v, nb[v], done)
        el = Eliminator()
        piv, ker = [], []
        for i, g in enumerate(gens):
            new, comb = el.add(g)
            if new:
                piv.append(i)
            else:
                ker.append(comb)
        steps.append(dict(v=v, r=r, rn=len(piv), rho=rho, piv=piv, ker=ker))
        B = [gens[i] for i in piv]
    assert not B, "state space must be empty at the end"
    return steps


def width(steps):
    """Largest table exponent of a plan (the in-place arena needs 2^width entries)."""
    return max(max(s["r"], s["rn"]) for s in steps) if steps else 0
