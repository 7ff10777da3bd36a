"""Dense statevector of a small circuit (n <= ~22): the brute-force checker of amplitudes and samples.

TEST INFRASTRUCTURE ONLY (part of the oracle): tests use it to check Born probabilities, as the reference's own tests
do with their statevector helpers (test_tableau.py:10-17 G1/apply1/cz).  Qubit 0 is the most significant bit of the
state index.  Gate matrices are the qelib1 definitions; ``u3``/``u`` is OpenQASM 2's U(theta, phi, lambda).
"""
import math
import re

import numpy as np

_SQ2 = math.sqrt(2)
G1 = {
    "h": np.array([[1, 1], [1, -1]]) / _SQ2,
    "s": np.diag([1, 1j]),
    "sdg": np.diag([1, -1j]),
    "sx": np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]]) / 2,
    "sxdg": np.array([[1 - 1j, 1 + 1j], [1 + 1j, 1 - 1j]]) / 2,
    "x": np.array([[0, 1], [1, 0]]),
    "z": np.diag([1, -1]),
    "t": np.diag([1, np.exp(1j * np.pi / 4)]),
    "tdg": np.diag([1, np.exp(-1j * np.pi / 4)]),
}


def _angles(arg):
    return [float(eval(a, {"__builtins__": {}}, {"pi": math.pi})) for a in arg.split(",")]


def gate(name):
    if name in G1:
        return G1[name]
    m = re.match(r"rz\((.*)\)$", name)
    if m:
        (th,) = _angles(m.group(1))
        return np.diag([np.exp(-0.5j * th), np.exp(0.5j * th)])
    m = re.match(r"(?:u3|u)\((.*)\)$", name)
    if m:
        th, ph, la = _angles(m.group(1))
        c, s = math.cos(th / 2), math.sin(th / 2)
        return np.array([[c, -np.exp(1j * la) * s], [np.exp(1j * ph) * s, np.exp(1j * (ph + la)) * c]])
    raise ValueError(name)


def dense_state(n, ops):
    psi = np.zeros([2] * n, complex)
    psi[(0,) * n] = 1
    for name, qs in ops:
        if name == "cz":
            idx = [slice(None)] * n
            idx[qs[0]] = 1
            idx[qs[1]] = 1
            psi[tuple(idx)] *= -1
        else:
            psi = np.moveaxis(np.tensordot(gate(name), psi, axes=([1], [qs[0]])), 0, qs[0])
    return psi.reshape(-1)


def probabilities(n, ops):
    return np.abs(dense_state(n, ops)) ** 2


def index_of(bits_by_qubit):
    """state index of a bitstring given per qubit (qubit 0 most significant)."""
    idx = 0
    for b in bits_by_qubit:
        idx = 2 * idx + int(b)
    return idx


def dense_state_torch(n, ops, device="cuda"):
    """The same statevector computed with torch (complex128) on `device`, for n up to ~28 (2^n x 16 bytes)."""
    import torch
    psi = torch.zeros([2] * n, dtype=torch.complex128, device=device)
    psi[(0,) * n] = 1
    for name, qs in ops:
        if name == "cz":
            idx = [slice(None)] * n
            idx[qs[0]] = 1
            idx[qs[1]] = 1
            psi[tuple(idx)] *= -1
        else:
            G = torch.tensor(gate(name), dtype=torch.complex128, device=device)
            psi = torch.movedim(torch.tensordot(G, psi, dims=([1], [qs[0]])), 0, qs[0])
    return psi.reshape(-1)
