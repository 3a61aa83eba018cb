"""Shared helpers of the GPU parity tests (seeded inputs and comparisons)."""
import numpy as np
import scipy.linalg as sl

import oracle as orc
from ecg_b200 import synth


def rel_err(a, b, floor=0.0):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def lowest_energy(o, K):
    """Lowest eigenvalue of the oracle's pencil (I-mode storage, lambda~ = 0)."""
    o.compute_mat_elem(1, K, 0.0)
    H = np.tril(o.H[:K, :K]) + np.tril(o.H[:K, :K], -1).conj().T
    return sl.eigh(H, o.S[:K, :K], eigvals_only=True)[0]


def problem(cfg, K, max_nfo=0):
    """(system, params, lambda~, oracle) for the first K functions of config cfg."""
    sysm, params = synth.config_basis(cfg, K=K)
    o = orc.Oracle(sysm, K, max_nfo=max_nfo)
    o.set_params(params)
    E0 = lowest_energy(o, K)
    return sysm, params, E0 * (1.0 + 1e-10), o


EPS = np.finfo(np.float64).eps


def _unpack(params, n):
    K = params.shape[0]
    np_ = n * (n + 1) // 2
    L = np.zeros((K, n, n))
    B = np.zeros((K, n, n))
    k = 0
    for i in range(n):
        for j in range(i, n):
            L[:, j, i] = params[:, k]
            B[:, j, i] = params[:, np_ + k]
            B[:, i, j] = params[:, np_ + k]
            k += 1
    return L, B


def term_conditions(sysm, pk, pl, terms):
    """cond(C) of each (bra, ket, permutation) term, C = Ck^* + P'ClP."""
    Lk, Bk = _unpack(np.atleast_2d(pk), sysm.n)
    Ll, Bl = _unpack(np.atleast_2d(pl), sysm.n)
    P = sysm.yhy_mats[np.asarray(terms)].astype(float)
    Pt = np.transpose(P, (0, 2, 1))
    C = (Lk @ np.transpose(Lk, (0, 2, 1)) - 1j * Bk) + Pt @ (Ll @ np.transpose(Ll, (0, 2, 1)) + 1j * Bl) @ P
    return np.linalg.cond(C)


def pair_conditions(sysm, params):
    """(K, K) array: for pair (k, l) the largest cond(C) over the Y^+Y terms
    and over the two diagonal terms that normalise it (f = 1/sqrt(S_kk S_ll))."""
    K = params.shape[0]
    kk, ll = np.meshgrid(np.arange(K), np.arange(K), indexing="ij")
    kk, ll = kk.ravel(), ll.ravel()
    kap = np.zeros(K * K)
    for t in range(sysm.T):
        kap = np.maximum(kap, term_conditions(sysm, params[kk], params[ll], np.full(kk.size, t)))
    kap = kap.reshape(K, K)
    dk = np.diag(kap).copy()
    return np.maximum(kap, np.maximum(dk[:, None], dk[None, :]))


def tolerance(kappa, rtol=1e-12, c=64.0):
    """Relative tolerance of a comparison between two FP64 evaluations of an
    element whose inputs pass through a matrix of condition number kappa:
    1e-12, or c * eps * kappa when the element is worse conditioned (both
    evaluations then carry errors of a few eps * kappa)."""
    return np.maximum(rtol, c * EPS * np.asarray(kappa))
