"""Stabilizer tableau of the Clifford body of a QASM circuit.

Drop-in for the reference's ``tableau.py`` (``parse`` tableau.py:9, ``Tableau`` tableau.py:21-37,
``clifford_body`` tableau.py:39-49, ``gf2_rank`` tableau.py:51-60, ``cut_rank`` tableau.py:62-66).

Representation.  The tableau of C|0> has n generators; generator i is the Pauli row (x_i, z_i) with sign bit r_i.
Every supported gate acts on one or two *columns* of the tableau at once, for all generators, so this module stores
the tableau column-wise as Python integers used as bit vectors over the generators:

    X[q] bit i  = x-part of generator i on qubit q,     Z[q] likewise,     sgn bit i = sign of generator i.

A gate is then a handful of big-integer operations regardless of n.  The update rules are the Aaronson-Gottesman
conjugation rules (sign flips where the conjugated Pauli picks up a minus sign), with ``sx`` = H S H and
``sxdg`` = H S^dag H up to a global phase, exactly as the reference applies them.  ``xs``, ``zs`` and ``r`` give the
same (n, n) / (n,) uint8 arrays the reference exposes (row = generator, column = qubit), and accept assignment.
"""
import re

import numpy as np

_CLIFFORD = ("h", "s", "sdg", "sx", "sxdg", "x", "z", "cz")


def _split_gate(line):
    """'name args' -> (name, args); a space inside the gate's parentheses does not split."""
    depth = 0
    for i, ch in enumerate(line):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == " " and depth == 0:
            return line[:i], line[i + 1:]
    return line, ""


def parse(path):
    """(n, [(name, [qubits])]) of an OPENQASM 2 file with one register ``q`` (reference tableau.py:9-19)."""
    n = None
    ops = []
    with open(path) as f:
        for raw in f:
            line = raw.strip().rstrip(";")
            if not line or line.startswith(("OPENQASM", "include")):
                continue
            reg = re.match(r"qreg q\[(\d+)\]", line)
            if reg:
                n = int(reg.group(1))
                continue
            name, args = _split_gate(line)
            ops.append((name.replace(" ", ""), [int(a) for a in re.findall(r"q\[(\d+)\]", args)]))
    return n, ops


def _bits_to_array(cols, n):
    """Column bit vectors over generators -> (n generators, n qubits) uint8 array."""
    out = np.zeros((n, n), np.uint8)
    for q, col in enumerate(cols):
        if col:
            rows = [i for i in range(n) if (col >> i) & 1]
            out[rows, q] = 1
    return out


def _array_to_bits(arr):
    arr = np.asarray(arr)
    n = arr.shape[1]
    return [int(sum(1 << int(i) for i in np.nonzero(arr[:, q] & 1)[0])) for q in range(n)]


class Tableau:
    """Stabilizer tableau, column-packed (see module docstring).  Methods mirror the reference's gate set."""

    def __init__(self, n):
        self.n = n
        self.X = [0] * n                       # C|0>: generator i = Z_i
        self.Z = [1 << q for q in range(n)]
        self.sgn = 0

    # --- array views (the reference's public attributes) ---
    @property
    def xs(self):
        return _bits_to_array(self.X, self.n)

    @xs.setter
    def xs(self, arr):
        self.X = _array_to_bits(arr)

    @property
    def zs(self):
        return _bits_to_array(self.Z, self.n)

    @zs.setter
    def zs(self, arr):
        self.Z = _array_to_bits(arr)

    @property
    def r(self):
        return np.array([(self.sgn >> i) & 1 for i in range(self.n)], np.uint8)

    @r.setter
    def r(self, arr):
        self.sgn = int(sum(1 << i for i, b in enumerate(np.asarray(arr)) if int(b) & 1))

    # --- gates ---
    def h(self, q):
        x, z = self.X[q], self.Z[q]
        self.sgn ^= x & z                      # Y -> -Y
        self.X[q], self.Z[q] = z, x

    def s_(self, q):
        x, z = self.X[q], self.Z[q]
        self.sgn ^= x & z                      # Y -> -X
        self.Z[q] = z ^ x

    def z(self, q):
        self.sgn ^= self.X[q]                  # X, Y anticommute with Z

    def x(self, q):
        self.sgn ^= self.Z[q]                  # Z, Y anticommute with X

    def sdg(self, q):
        self.z(q)
        self.s_(q)

    def sx(self, q):                           # H S H = sqrt(X) up to a global phase
        self.h(q)
        self.s_(q)
        self.h(q)

    def sxdg(self, q):                         # H S^dag H
        self.h(q)
        self.sdg(q)
        self.h(q)

    def cz(self, a, b):
        xa, xb, za, zb = self.X[a], self.X[b], self.Z[a], self.Z[b]
        self.sgn ^= xa & xb & (za ^ zb)
        self.Z[a] = za ^ xb
        self.Z[b] = zb ^ xa

    def apply(self, name, qs):
        if name == "cz":
            self.cz(*qs)
            return
        table = {"h": self.h, "s": self.s_, "sdg": self.sdg, "sx": self.sx, "sxdg": self.sxdg, "x": self.x, "z": self.z}
        if name not in table:
            raise KeyError(name)
        table[name](*qs)

    def copy(self):
        t = Tableau.__new__(Tableau)
        t.n, t.X, t.Z, t.sgn = self.n, list(self.X), list(self.Z), self.sgn
        return t


def clifford_body(path):
    """(n, tableau of the leading Clifford gates, remaining tail ops) (reference tableau.py:39-49)."""
    n, ops = parse(path)
    T = Tableau(n)
    i = len(ops)
    for j, (name, qs) in enumerate(ops):
        if name not in _CLIFFORD:
            i = j
            break
        T.apply(name, qs)
    return n, T, ops[i:]


def rank_of_ints(vecs):
    """GF(2) rank of a list of bit vectors (Python ints)."""
    piv = {}                                   # leading bit -> vector
    for v in vecs:
        while v:
            hb = v.bit_length() - 1
            if hb not in piv:
                piv[hb] = v
                break
            v ^= piv[hb]
    return len(piv)


def gf2_rank(M):
    """GF(2) rank of a 0/1 matrix (reference tableau.py:51-60)."""
    M = np.asarray(M)
    if M.ndim != 2 or M.size == 0:
        return 0
    rows = [int(sum(1 << j for j in np.nonzero(row & 1)[0])) for row in M]
    return rank_of_ints(rows)


def cut_rank(T, A):
    """Entanglement in ebits across A | complement: rank of the generators restricted to B, minus |B|
    (reference tableau.py:62-66)."""
    B = sorted(set(range(T.n)) - set(A))
    xs, zs = T.xs, T.zs
    G = np.concatenate([xs[:, B], zs[:, B]], axis=1)
    return gf2_rank(G) - len(B)
