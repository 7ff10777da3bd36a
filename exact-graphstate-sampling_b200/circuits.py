"""Seeded circuit families of the benchmark workloads (Clifford body + one single-qubit rotation layer).

* ``graph_state_circuit(n, p, seed)``: H on every qubit, CZ on the edges of a seeded G(n, p), a uniformly random
  single-qubit Clifford per qubit (one of the 24), then a U3 layer with theta, phi, lambda uniform in [0, 2 pi).
* ``matching_circuit(n, depth, seed)``: H on every qubit, then ``depth`` layers of CZ on a seeded uniformly random
  perfect matching (odd n leaves one qubit idle per layer), each followed by seeded random single-qubit Cliffords,
  then a Haar-random U3 per qubit (theta = 2 arccos sqrt(u), phi, lambda uniform).
* ``brickwork_circuit(n, seed)``: the reference's IBM-like construction (frontier.py:12-20): alternating
  nearest-neighbour CZ brickwork of depth n with S^b SX on every qubit after each layer.

Circuits are lists of (gate, [qubits]) ops; ``tableau_of`` builds the Clifford body's tableau and ``to_qasm`` writes
OPENQASM 2 text that ``tableau.clifford_body`` reads back.
"""
import math

import numpy as np

from tableau import Tableau

_H = np.array([[1, 1], [1, -1]]) / math.sqrt(2)
_S = np.diag([1, 1j])


def _canon(U):
    """2x2 unitary up to global phase -> hashable key."""
    flat = U.reshape(-1)
    i = int(np.argmax(np.abs(flat) > 1e-9))
    ph = flat[i] / abs(flat[i])
    V = U / ph
    return tuple(np.round(V.real, 9).reshape(-1)) + tuple(np.round(V.imag, 9).reshape(-1))


def _clifford_words():
    """The 24 single-qubit Cliffords as shortest words over {h, s} (applied left to right), breadth first."""
    seen = {_canon(np.eye(2)): ()}
    frontier = [((), np.eye(2, dtype=complex))]
    while frontier:
        nxt = []
        for word, U in frontier:
            for g, G in (("h", _H), ("s", _S)):
                V = G @ U
                key = _canon(V)
                if key not in seen:
                    seen[key] = word + (g,)
                    nxt.append((word + (g,), V))
        frontier = nxt
    words = sorted(seen.values(), key=lambda w: (len(w), w))
    assert len(words) == 24
    return words


CLIFFORD_WORDS = _clifford_words()


def random_clifford_ops(q, rng):
    return [(g, [q]) for g in CLIFFORD_WORDS[int(rng.integers(24))]]


def u3_op(q, theta, phi, lam):
    return (f"u3({theta!r},{phi!r},{lam!r})", [q])


def graph_state_circuit(n, p=0.5, seed=0):
    rng = np.random.default_rng(seed)
    body = [("h", [q]) for q in range(n)]
    for i in range(n):
        for j in range(i + 1, n):
            if rng.random() < p:
                body.append(("cz", [i, j]))
    for q in range(n):
        body += random_clifford_ops(q, rng)
    tail = [u3_op(q, *(float(x) for x in rng.uniform(0, 2 * math.pi, 3))) for q in range(n)]
    return n, body, tail


def haar_u3(rng):
    theta = 2 * math.acos(math.sqrt(float(rng.random())))
    phi, lam = (float(x) for x in rng.uniform(0, 2 * math.pi, 2))
    return theta, phi, lam


def matching_circuit(n, depth=None, seed=0):
    depth = n if depth is None else depth
    rng = np.random.default_rng(seed)
    body = [("h", [q]) for q in range(n)]
    for _ in range(depth):
        perm = rng.permutation(n)
        for a in range(0, n - 1, 2):
            i, j = int(perm[a]), int(perm[a + 1])
            body.append(("cz", [min(i, j), max(i, j)]))
        for q in range(n):
            body += random_clifford_ops(q, rng)
    tail = [u3_op(q, *haar_u3(rng)) for q in range(n)]
    return n, body, tail


def brickwork_circuit(n, seed, tail_theta=0.9553166181245092):
    """IBM-like brickwork instance with the reference's measurement tail tdg; h; rz(theta); h."""
    import random
    rng = random.Random(seed)
    body = [("h", [q]) for q in range(n)]
    for layer in range(n):
        for a in range(layer % 2, n - 1, 2):
            body.append(("cz", [a, a + 1]))
        for q in range(n):
            if rng.random() < 0.5:
                body.append(("s", [q]))
            body.append(("sx", [q]))
    tail = []
    for q in range(n):
        tail += [("tdg", [q]), ("h", [q]), (f"rz({tail_theta})", [q]), ("h", [q])]
    return n, body, tail


def tableau_of(n, body):
    T = Tableau(n)
    for name, qs in body:
        T.apply(name, qs)
    return T


def to_qasm(n, body, tail):
    lines = ["OPENQASM 2.0;", 'include "qelib1.inc";', f"qreg q[{n}];"]
    for name, qs in list(body) + list(tail):
        lines.append(name + " " + ",".join(f"q[{q}]" for q in qs) + ";")
    return "\n".join(lines) + "\n"

