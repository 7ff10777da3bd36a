"""Exact amplitudes <b| W (x) |S> of a circuit = Clifford body + per-qubit single-qubit tail.

Drop-in for the reference's ``amp.py`` (``tail_matrix`` amp.py:7-17, ``Amplitudes`` amp.py:19-29).  With
(U_0 x ... x U_{n-1}) |S> = e^{i phi} |G_A> from the graph form, each qubit's rotation folds into the 2x2 matrix
M_j = W_j U_j^dag, and  <b|psi> = 2^{-n/2} sum_x prod_j M_j[b_j, x_j] (-1)^{x^T A x}.

Gate matrices are built with the same numpy expressions as the reference so that M (and the plan text, which prints
M with %.17g) match bit for bit.  Beyond the reference's tail gates (h, t, tdg, rz) this module also accepts the
OpenQASM 2 ``u3(theta, phi, lambda)`` / ``u(...)`` gate, which the rotation layers of the benchmark circuits use;
any other name still raises ValueError as in the reference.
"""
import math
import re

import numpy as np

from graphform import graph_form
from plan import plan

_NUM = re.compile(r"^[\s0-9eE+\-*/().pi]*$")


def _angle(text):
    """float of an angle expression: a number or an arithmetic expression in numbers and pi."""
    try:
        return float(text)
    except ValueError:
        if not _NUM.match(text):
            raise ValueError(f"bad angle {text!r}")
        return float(eval(text, {"__builtins__": {}}, {"pi": math.pi}))


def u3_matrix(theta, phi, lam):
    """OpenQASM 2 U(theta, phi, lambda) = Rz(phi) Ry(theta) Rz(lambda) up to a global phase."""
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    return np.array([[c, -np.exp(1j * lam) * s], [np.exp(1j * phi) * s, np.exp(1j * (phi + lam)) * c]])


def gate_matrix(name):
    if name == "h":
        return np.array([[1, 1], [1, -1]]) / np.sqrt(2)
    if name == "tdg":
        return np.diag([1, np.exp(-1j * np.pi / 4)])
    if name == "t":
        return np.diag([1, np.exp(1j * np.pi / 4)])
    m = re.match(r"rz\((.*)\)$", name)
    if m:
        th = _angle(m.group(1))
        return np.diag([np.exp(-1j * th / 2), np.exp(1j * th / 2)])
    m = re.match(r"(?:u3|u)\((.*)\)$", name)
    if m:
        parts = [p.strip() for p in m.group(1).split(",")]
        if len(parts) != 3:
            raise ValueError(f"unsupported tail gate {name}")
        return u3_matrix(*(_angle(p) for p in parts))
    raise ValueError(f"unsupported tail gate {name}")


def tail_matrix(ops):
    """Product of a qubit's tail gates, first gate rightmost (reference amp.py:7-17)."""
    M = np.eye(2, dtype=complex)
    for name, _ in ops:
        M = gate_matrix(name) @ M
    return M


class Amplitudes:
    """Graph form, per-qubit matrices M_j and the out-of-place plan of a Clifford body + single-qubit tail."""

    def __init__(self, n, T, tail, order=None):
        self.n = n
        self.A, U = graph_form(T)
        per = [[] for _ in range(n)]
        for name, qs in tail:
            assert len(qs) == 1, "tail must be single-qubit"
            per[qs[0]].append((name, qs))
        self.W = [tail_matrix(per[q]) for q in range(n)]
        self.M = [self.W[q] @ U[q].conj().T for q in range(n)]
        self.order = order or list(range(n))
        self.steps = plan(self.A, self.order)

    def weights(self, b):
        """(M_q[b_q, 0], M_q[b_q, 1]) per qubit for the output string b (qubit order)."""
        return [(self.M[q][b[q], 0], self.M[q][b[q], 1]) for q in range(self.n)]
