"""Exact ground-state energies of the shipped models (independent physics checks).

TEST INFRASTRUCTURE ONLY.

- Kitaev chain (reference src/operators.cpp:394-431, H_Kitaev(t, p, u)):
  H = sum_i [t c+_i c_{i+1} - p c_i c_{i+1} + h.c.] - 2u sum_i n_i, open chain.
  Free fermions: with A = tridiag(t; -2u) and B antisymmetric, B[i,i+1] = p, the
  BdG matrix [[A, B], [-B, -A]] has eigenvalues +-eps_k and the ground energy is
  E0 = Tr(A)/2 - sum_{eps>0} eps / 2.  Its fermion parity depends on the signs
  of the Pfaffian; for |u| < |t| the even/odd splitting is ~ (u/t)^L.
- XYZ chain (src/operators.cpp:352-391, H_XYZ(jx, jy, jz), Pauli matrices):
  H = sum_i jx X_i X_{i+1} + jy Y_i Y_{i+1} + jz Z_i Z_{i+1}; sector 0 of the
  reference's Z2 label = even number of down spins.
- 3-state Potts (src/operators.cpp:290-350, H_Potts3(f, j, 0, 0)):
  H = -f sum_i (T_i + T_i^+) - j sum_i (S_i S^+_{i+1} + S^+_i S_{i+1}),
  T = diag(1, w, w^2), S|q> = |q-1> (shift), Z3 charge = sum of labels mod 3.
"""
from __future__ import annotations

import numpy as np


def kitaev_bdg(L: int, t: float, p: float, u: float) -> float:
    A = np.zeros((L, L))
    B = np.zeros((L, L))
    for i in range(L):
        A[i, i] = -2 * u
    for i in range(L - 1):
        A[i, i + 1] = A[i + 1, i] = t
        B[i, i + 1] = p
        B[i + 1, i] = -p
    H = np.block([[A, B], [-B, -A]])
    w = np.linalg.eigvalsh(H)
    return float(0.5 * np.trace(A) - 0.5 * w[w > 0].sum())


def _kron_chain(ops):
    out = ops[0]
    for o in ops[1:]:
        out = np.kron(out, o)
    return out


def xyz_ed(L: int, jx: float, jy: float, jz: float, sector: int = 0,
           periodic: bool = False) -> float:
    """periodic adds the bond (L-1, 0), the reference's PBC build (xyz.cpp:39-42)."""
    X = np.array([[0, 1], [1, 0]], complex)
    Y = np.array([[0, -1j], [1j, 0]], complex)
    Z = np.array([[1, 0], [0, -1]], complex)
    I = np.eye(2)
    H = np.zeros((2 ** L, 2 ** L), complex)
    for i in range(L if periodic else L - 1):
        for J, P in ((jx, X), (jy, Y), (jz, Z)):
            ops = [I] * L
            ops[i] = P
            ops[(i + 1) % L] = P
            H += J * _kron_chain(ops)
    # basis state index bits: label 1 = down spin; keep even/odd count of 1s
    idx = [s for s in range(2 ** L) if bin(s).count("1") % 2 == sector]
    return float(np.linalg.eigvalsh(H[np.ix_(idx, idx)])[0])


def potts_ed(L: int, f: float, j: float, sector: int = 0, periodic: bool = False) -> float:
    """periodic adds the bond (L-1, 0) without a second field term, the reference's
    PBC build (potts.cpp:44-47: edge operators H_Potts3(0, j, p, t))."""
    w = np.exp(2j * np.pi / 3)
    T = np.diag([1, w, w * w])
    S = np.zeros((3, 3), complex)
    for q in range(3):
        S[(q - 1) % 3, q] = 1.0
    I = np.eye(3)
    D = 3 ** L
    H = np.zeros((D, D), complex)
    for i in range(L):
        ops = [I] * L
        ops[i] = T + T.conj().T
        H += -f * _kron_chain(ops)
    for i in range(L if periodic else L - 1):
        ops = [I] * L
        ops[i] = S
        ops[(i + 1) % L] = S.conj().T
        M = _kron_chain(ops)
        H += -j * (M + M.conj().T)
    charge = []
    for s in range(D):
        q, x = 0, s
        for _ in range(L):
            q += x % 3
            x //= 3
        charge.append(q % 3)
    idx = [s for s in range(D) if charge[s] == sector]
    return float(np.linalg.eigvalsh(H[np.ix_(idx, idx)])[0])
