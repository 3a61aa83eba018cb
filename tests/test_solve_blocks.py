"""Block form of LDLHS's two triangular solves (src/linalg.f90:618-775) as
the cooperative solve kernels run it (csrc/invit.cu, k_fwd_coop /
k_bwd_coop): panel j applies its inverse unit-lower diagonal block
Linv_j = (U_jj^H)^-1 to its right-hand side minus the panels it depends
on, except the neighbouring panel, whose term comes in afterwards through
the products k_ldl_mn precomputes, M_j = Linv_j U(j-1, j)^H (forward) and
N_j = Linv_j^H U(j, j+1) (backward).  Checked here in numpy against a
dense solve of U^H D U x = w, with 64-row panels and with the irregular
panel boundaries a bordered factorisation leaves."""
import numpy as np
import pytest


def ldlh(M):
    """Unit upper U and pivots d with M = U^H diag(d) U (no pivoting)."""
    n = M.shape[0]
    A = M.copy()
    U = np.eye(n, dtype=complex)
    d = np.zeros(n, dtype=complex)
    for q in range(n):
        d[q] = A[q, q].real
        U[q, q + 1:] = A[q, q + 1:] / d[q]
        A[q + 1:, q + 1:] -= np.outer(np.conj(U[q, q + 1:]), A[q, q + 1:])
    return U, d


def block_solve(U, d, w, starts):
    n = U.shape[0]
    b = list(starts) + [n]
    nb = len(starts)
    sl = [slice(b[j], b[j + 1]) for j in range(nb)]
    Linv = [np.linalg.inv(U[s, s].conj().T) for s in sl]
    Mf = [None] + [Linv[j] @ U[sl[j - 1], sl[j]].conj().T for j in range(1, nb)]
    Nb = [Linv[j].conj().T @ U[sl[j], sl[j + 1]] for j in range(nb - 1)] + [None]
    y = np.zeros(n, dtype=complex)
    for j in range(nb):  # forward: y_j = Linv_j (w_j - sum_{a<j-1} U(a,j)^H y_a) - M_j y_{j-1}
        acc = sum((U[sl[a], sl[j]].conj().T @ y[sl[a]] for a in range(j - 1)), np.zeros(b[j + 1] - b[j], complex))
        y[sl[j]] = Linv[j] @ (w[sl[j]] - acc)
        if j > 0:
            y[sl[j]] -= Mf[j] @ y[sl[j - 1]]
    z = y / d
    x = np.zeros(n, dtype=complex)
    for j in reversed(range(nb)):  # backward: x_j = Linv_j^H (z_j - sum_{c>j+1} U(j,c) x_c) - N_j x_{j+1}
        acc = sum((U[sl[j], sl[c]] @ x[sl[c]] for c in range(j + 2, nb)), np.zeros(b[j + 1] - b[j], complex))
        x[sl[j]] = Linv[j].conj().T @ (z[sl[j]] - acc)
        if j + 1 < nb:
            x[sl[j]] -= Nb[j] @ x[sl[j + 1]]
    return x


@pytest.mark.parametrize("n,starts", [
    (300, None),                          # 64-row panels, short last panel
    (64, None),                           # one panel
    (260, [0, 64, 100, 164, 228]),        # a truncated panel, as after a bordered step
])
def test_block_solve_with_neighbour_products(n, starts):
    rng = np.random.default_rng(n)
    X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    M = X @ X.conj().T / n + np.diag(rng.uniform(-2.0, 2.0, n))  # Hermitian, indefinite
    U, d = ldlh(M)
    w = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    if starts is None:
        starts = list(range(0, n, 64))
    x = block_solve(U, d, w, starts)
    ref = np.linalg.solve(U.conj().T @ np.diag(d) @ U, w)
    assert np.max(np.abs(x - ref)) <= 1e-9 * np.max(np.abs(ref))
