"""The oracle's two LDLHF branches (src/linalg.f90:356-452): the parallel
branch, with the OpenMP threads as the MPI ranks, factorises the same matrix
as the serial branch to rounding, from scratch and as a bordered update
(m > 1), and reports the same zero pivot."""
import numpy as np
import pytest

import oracle as orc


def _hermitian_pd(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return X @ X.conj().T / n + np.eye(n)


def _factor(A, m, fn, invD=None):
    n = A.shape[0]
    M = np.asfortranarray(A.copy())
    invD = np.zeros(n, dtype=np.complex128) if invD is None else invD.copy()
    w = np.zeros(n, dtype=np.complex128)
    err = fn(m, n, M.ctypes.data_as(orc._dp), n, invD.ctypes.data_as(orc._dp), w.ctypes.data_as(orc._dp))
    return M, invD, err


@pytest.mark.parametrize("threads", [3, 8])
@pytest.mark.parametrize("n,m", [(97, 1), (160, 1), (160, 121)])
def test_parallel_branch_matches_serial(n, m, threads):
    lib = orc.load()
    t0 = orc.get_threads()
    orc.set_threads(threads)
    try:
        A = np.tril(_hermitian_pd(n, n + m))  # the lower triangle holds the matrix
        pre = None
        if m > 1:  # factor of the leading m-1 rows from the serial branch
            Ms, inv0, err0 = _factor(A, 1, lib.orc_ldlhf)
            assert err0 == 0
            pre = (np.triu(Ms[:, :m - 1], 1) + np.tril(A[:, :m - 1]), inv0)
            A = A.copy()
            A[:, :m - 1] = pre[0]
        Ms, invs, es = _factor(A, m, lib.orc_ldlhf, None if pre is None else pre[1])
        Mp, invp, ep = _factor(A, m, lib.orc_ldlhf_par, None if pre is None else pre[1])
        assert es == ep == 0
        U = np.triu(Ms, 1)
        assert np.max(np.abs(np.triu(Mp, 1) - U)) <= 1e-12 * max(np.max(np.abs(U)), 1.0)
        assert np.max(np.abs(invp - invs)) <= 1e-12 * np.max(np.abs(invs))
        assert np.array_equal(np.tril(Mp), np.tril(A))  # the lower triangle is left as it was
    finally:
        orc.set_threads(t0)


def test_parallel_branch_zero_pivot():
    lib = orc.load()
    t0 = orc.get_threads()
    orc.set_threads(4)
    try:
        n = 40
        A = np.zeros((n, n), dtype=np.complex128)
        A[np.arange(n), np.arange(n)] = 1.0
        A[17, 17] = 0.0  # exactly zero pivot in row 18
        _, _, es = _factor(A, 1, lib.orc_ldlhf)
        _, _, ep = _factor(A, 1, lib.orc_ldlhf_par)
        assert es == ep == 1
    finally:
        orc.set_threads(t0)
