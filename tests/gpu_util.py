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


def pair_conditions_at(sysm, params, kk, ll):
    """pair_conditions for the listed pairs only (arrays of 0-based k, l)."""
    kk = np.asarray(kk)
    ll = np.asarray(ll)
    kap = np.zeros(kk.size)
    for a, b in ((kk, ll), (kk, kk), (ll, ll)):
        for t in range(sysm.T):
            kap = np.maximum(kap, term_conditions(sysm, params[a], params[b], np.full(a.size, t)))
    return kap


def hs_ratio(o, sysm, params, K, lam, method, H, S, dS):
    """Largest |GPU - oracle| / (scale * tolerance) over every stored element
    of H, S (lower triangle; strict in 'G' storage) and diagS.  scale is the
    sum over Y^+Y terms of |coef| |term| as stored (terms of opposite sign
    cancel), plus |lambda~| times that of S for 'I' storage's H - lambda~ S;
    tolerance is 1e-12, or 64 eps cond(C) for the elements where that is
    larger (cond(C) evaluated only where an element is beyond 1e-12)."""
    lo = np.tril_indices(K, -1 if method == "G" else 0)
    aH, aS = o.term_magnitudes(K)
    f = 1.0 / np.sqrt(np.outer(o.diagS[:K], o.diagS[:K]))
    sH = ((aH + (abs(lam) * aS if method == "I" else 0.0)) * f)[lo]
    sS = (aS * f)[lo]
    dH = np.abs(H[lo] - o.H[:K, :K][lo]) / sH
    dSm = np.abs(S[lo] - o.S[:K, :K][lo]) / sS
    out = {"H_within_1e-12": float(np.mean(dH <= 1e-12)), "S_within_1e-12": float(np.mean(dSm <= 1e-12))}
    for name, d in (("H", dH), ("S", dSm)):
        bad = np.nonzero(d > 1e-12)[0]
        r = float(np.max(d)) / 1e-12 if d.size else 0.0
        if bad.size:
            kap = pair_conditions_at(sysm, params, lo[0][bad], lo[1][bad])
            r = max(float(np.max(np.where(d <= 1e-12, d, 0.0))) / 1e-12, float(np.max(d[bad] / tolerance(kap))))
        out[name] = r
    dd = np.abs(dS - o.diagS[:K]) / np.abs(o.diagS[:K])
    bad = np.nonzero(dd > 1e-12)[0]
    rd = float(np.max(dd)) / 1e-12
    if bad.size:
        kap = pair_conditions_at(sysm, params, bad, bad)
        rd = max(float(np.max(np.where(dd <= 1e-12, dd, 0.0))) / 1e-12, float(np.max(dd[bad] / tolerance(kap))))
    out["diagS"] = rd
    return out
