"""Local-Clifford-equivalent graph form of a stabilizer state.

Drop-in for the reference's ``graphform.py`` (``graph_form`` graphform.py:21-50, ``_rowmul`` graphform.py:11-19).
``graph_form(T)`` returns ``(A, U)``: A the symmetric 0/1 adjacency matrix (uint8) and U a list of per-qubit 2x2
unitaries with (U_0 x ... x U_{n-1}) |S> = e^{i phi} |G_A>.

The procedure has to make the same choices as the reference, because A and the floating-point U_j feed the plan
and the rotation matrices M_j = W_j U_j^dag bit for bit:
  1. Hadamards, greedily in qubit order over at most three sweeps, each kept only if it raises the rank of the X
     block (a rejected Hadamard is undone by a second Hadamard, and both enter U_j);
  2. Gauss-Jordan reduction of the X block to the identity with sign-exact generator products;
  3. S^dag on every qubit whose generator has a Y on the diagonal, then Z on every generator with a minus sign.
Step 1 runs on the column-packed tableau; steps 2-3 on generator rows packed as bit vectors over qubits.
"""
import numpy as np

from tableau import Tableau, rank_of_ints

MAT = {"h": np.array([[1, 1], [1, -1]]) / np.sqrt(2), "sdg": np.diag([1, -1j]), "z": np.diag([1, -1])}


def _popc(v):
    return bin(v).count("1")


def _product_phase(xk, zk, xi, zi):
    """Sum over qubits of the Aaronson-Gottesman g(x_k, z_k, x_i, z_i) (the power of i picked up by P_k P_i)."""
    y1 = xk & zk
    x1 = xk & ~zk
    z1 = zk & ~xk
    return (_popc(y1 & zi) - _popc(y1 & xi)
            + _popc(x1 & zi & xi) - _popc(x1 & zi & ~xi)
            + _popc(z1 & xi & ~zi) - _popc(z1 & xi & zi))


class _Rows:
    """Generator rows: x[i], z[i] bit vectors over qubits, s[i] sign bit."""

    def __init__(self, T):
        n = T.n
        self.n = n
        self.x = [0] * n
        self.z = [0] * n
        for q in range(n):
            cx, cz = T.X[q], T.Z[q]
            for i in range(n):
                if (cx >> i) & 1:
                    self.x[i] |= 1 << q
                if (cz >> i) & 1:
                    self.z[i] |= 1 << q
        self.s = [(T.sgn >> i) & 1 for i in range(n)]

    def mul_into(self, i, k):
        """generator i <- generator k * generator i, with the exact sign (reference graphform.py:11-19)."""
        ph = (2 * self.s[k] + 2 * self.s[i] + _product_phase(self.x[k], self.z[k], self.x[i], self.z[i])) % 4
        assert ph in (0, 2)
        self.s[i] = ph // 2
        self.x[i] ^= self.x[k]
        self.z[i] ^= self.z[k]

    def sdg(self, q):                          # Z then S on column q
        b = 1 << q
        for i in range(self.n):
            xb = (self.x[i] & b) != 0
            zb = (self.z[i] & b) != 0
            self.s[i] ^= int(xb)               # z(q)
            self.s[i] ^= int(xb and zb)        # s(q): Y -> -X
            if xb:
                self.z[i] ^= b

    def zgate(self, q):
        b = 1 << q
        for i in range(self.n):
            if self.x[i] & b:
                self.s[i] ^= 1


def graph_form(T0):
    n = T0.n
    T = T0.copy() if isinstance(T0, Tableau) else _from_arrays(T0)
    gates = []

    def xrank():
        return rank_of_ints(T.X)

    # 1. Hadamards until the X block is invertible
    for _ in range(3):
        for j in range(n):
            if xrank() == n:
                break
            before = xrank()
            T.h(j)
            gates.append(("h", j))
            if xrank() <= before:
                T.h(j)
                gates.append(("h", j))
    assert xrank() == n, "could not make the X block invertible"

    # 2. reduce the X block to the identity
    R = _Rows(T)
    for c in range(n):
        cb = 1 << c
        p = next(i for i in range(c, n) if R.x[i] & cb)
        if p != c:
            R.x[c], R.x[p] = R.x[p], R.x[c]
            R.z[c], R.z[p] = R.z[p], R.z[c]
            R.s[c], R.s[p] = R.s[p], R.s[c]
        for i in range(n):
            if i != c and R.x[i] & cb:
                R.mul_into(i, c)

    # 3. clear Y on the diagonal, then the signs
    for i in range(n):
        if (R.z[i] >> i) & 1:
            R.sdg(i)
            gates.append(("sdg", i))
    for i in range(n):
        if R.s[i]:
            R.zgate(i)
            gates.append(("z", i))

    A = np.zeros((n, n), np.uint8)
    for i in range(n):
        assert R.x[i] == 1 << i and R.s[i] == 0 and not (R.z[i] >> i) & 1
        for j in range(n):
            if (R.z[i] >> j) & 1:
                A[i, j] = 1
    assert (A == A.T).all()
    U = [np.eye(2, dtype=complex) for _ in range(n)]
    for g, q in gates:
        U[q] = MAT[g] @ U[q]
    return A, U


def _from_arrays(T0):
    """Accept any object with n, xs, zs, r (e.g. the reference's own Tableau)."""
    T = Tableau(T0.n)
    T.xs, T.zs, T.r = T0.xs, T0.zs, T0.r
    return T
