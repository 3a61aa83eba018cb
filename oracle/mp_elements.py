"""High-precision (mpmath) restatement of the energy part of MatrixElements
(src/matelem.f90:109-299): overlap S, kinetic T and Coulomb V of one pair
term, computed with 50 significant digits from the same formulas.

TEST INFRASTRUCTURE ONLY.  It pins the FP64 oracle and the GPU on single
pair terms: both must sit within their conditioning error (a small multiple
of eps * cond(C)) of these values.
"""
import mpmath as mp
import numpy as np

mp.mp.dps = 50


def _vech_to(n, v, lower=True):
    M = mp.matrix(n, n)
    k = 0
    for i in range(n):
        for j in range(i, n):
            M[j, i] = mp.mpf(float(v[k]))
            if not lower:
                M[i, j] = M[j, i]
            k += 1
    return M


def term_energy(pk, pl, P, mass_matrix, charges):
    """(H, S) of one (bra, ket, permutation) term at 50 digits."""
    n = len(P)
    np_ = n * (n + 1) // 2
    Lk = _vech_to(n, pk[:np_])
    Ll = _vech_to(n, pl[:np_])
    Bk = _vech_to(n, pk[np_:], lower=False)
    Bl = _vech_to(n, pl[np_:], lower=False)
    Pm = mp.matrix([[int(P[i][j]) for j in range(n)] for i in range(n)])
    Ak = Lk * Lk.T
    Al = Pm.T * (Ll * Ll.T) * Pm
    Blp = Pm.T * Bl * Pm
    Ck = mp.matrix(n, n)
    tCl = mp.matrix(n, n)
    for i in range(n):
        for j in range(n):
            Ck[i, j] = mp.mpc(Ak[i, j], -Bk[i, j])
            tCl[i, j] = mp.mpc(Al[i, j], Blp[i, j])
    C = Ck + tCl
    # principal-branch powers taken exactly as the reference: det C as the
    # product of the pseudo-Cholesky pivots, sqrt of the quotient
    G = mp.matrix(n, n)
    det = mp.mpc(1)
    for i in range(n):
        for j in range(i, n):
            s = C[i, j]
            for k in range(i - 1, -1, -1):
                s -= G[i, k] * G[j, k]
            if i == j:
                G[i, i] = mp.sqrt(s)
                det *= s
            else:
                G[j, i] = s / G[i, i]
    inv = C ** -1
    detL = abs(mp.fprod([Lk[i, i] for i in range(n)]) * mp.fprod([Ll[i, i] for i in range(n)]))
    c = detL / det
    S = mp.mpf(2) ** (mp.mpf(3 * n) / 2) * c * mp.sqrt(c)
    Mm = mp.matrix([[mp.mpf(float(mass_matrix[i][j])) for j in range(n)] for i in range(n)])
    W = tCl * inv * Ck
    T = 6 * S * sum(Mm[i, k] * W[k, i] for i in range(n) for k in range(n))
    q0 = mp.mpf(float(charges[0]))
    q = [mp.mpf(float(x)) for x in charges[1:]]
    cn = 2 / mp.sqrt(mp.pi) * S
    V = q0 * sum(q[i] * cn / mp.sqrt(inv[i, i]) for i in range(n))
    for i in range(n):
        for j in range(i + 1, n):
            V += q[i] * q[j] * cn / mp.sqrt(inv[i, i] + inv[j, j] - 2 * inv[j, i])
    return complex(T + V), complex(S)


def term_condition(pk, pl, P):
    """2-norm condition number of C = Ck^* + P'ClP, the matrix whose
    pseudo-Cholesky factor and inverse every element goes through."""
    n = len(P)
    np_ = n * (n + 1) // 2

    def unpack(v):
        L = np.zeros((n, n))
        B = np.zeros((n, n))
        k = 0
        for i in range(n):
            for j in range(i, n):
                L[j, i] = v[k]
                B[j, i] = B[i, j] = v[np_ + k]
                k += 1
        return L, B

    Lk, Bk = unpack(pk)
    Ll, Bl = unpack(pl)
    P = np.asarray(P, dtype=float)
    C = (Lk @ Lk.T - 1j * Bk) + P.T @ (Ll @ Ll.T + 1j * Bl) @ P
    return np.linalg.cond(C)
