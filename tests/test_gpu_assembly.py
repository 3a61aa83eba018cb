"""ComputeMatElem / ComputeMatElemAndDeriv + StoreHS / StoreHSD on the GPU
against the oracle: every stored element of H, S, diagS, diagH and Glob_D."""
import numpy as np
import pytest

import oracle as orc
from ecg_b200 import Context, synth
from gpu_util import pair_conditions, tolerance

pytestmark = pytest.mark.gpu


def _term_magnitudes(o, sysm, params):
    """(K, K) arrays of sum_t |coef_t| |H_t| and sum_t |coef_t| |S_t|."""
    K = params.shape[0]
    aH = np.zeros((K, K))
    aS = np.zeros((K, K))
    for k in range(K):
        for l in range(k + 1):
            for t in range(sysm.T):
                h, s, _, _ = o.matrix_elements(params[k], params[l], sysm.yhy_mats[t], 0)
                c = abs(sysm.yhy_coeffs[t])
                aH[k, l] += c * abs(h)
                aS[k, l] += c * abs(s)
    return aH, aS


def _ratio(a, b, scale, tol):
    """max over elements of |a - b| / (scale * tol)."""
    return float(np.max(np.abs(a - b) / (scale * tol)))


@pytest.mark.parametrize("cfg,K", [(0, 150), (1, 130), (4, 70)])
@pytest.mark.parametrize("method", ["I", "G"])
def test_hs_matches_oracle(cfg, K, method):
    sysm, params = synth.config_basis(cfg, K=K)
    lam = -0.55 if cfg == 0 else -1.1
    o = orc.Oracle(sysm, K)
    o.set_params(params)
    o.compute_mat_elem(1, K, lam, method=method)
    with Context(sysm, K, method=method) as ctx:
        ctx.set_params(params)
        ctx.compute_mat_elem(1, K, lam)
        H, S, dS, dH, _ = ctx.matrices(K)
    lo = np.tril_indices(K, -1 if method == "G" else 0)
    tol = tolerance(pair_conditions(sysm, params))[lo]
    Ho, So = o.H[:K, :K][lo], o.S[:K, :K][lo]
    # scale of each stored element: the sum over Y^+Y terms of |coef| times
    # the term's magnitude (terms of opposite sign cancel), normalised as
    # stored; H - lambda~ S also carries the rounding of lambda~ S
    aH, aS = _term_magnitudes(o, sysm, params)
    f = 1.0 / np.sqrt(np.outer(o.diagS[:K], o.diagS[:K]))
    sH = ((aH + (abs(lam) * aS if method == "I" else 0.0)) * f)[lo]
    sS = (aS * f)[lo]
    rH = _ratio(H[lo], Ho, sH, tol)
    rS = _ratio(S[lo], So, sS, tol)
    rd = _ratio(dS, o.diagS[:K], np.abs(o.diagS[:K]), np.diag(tolerance(pair_conditions(sysm, params))))
    tight = np.mean(np.abs(H[lo] - Ho) <= 1e-12 * sH)
    print(f"cfg {cfg} {method}: diff/tol H {rH:.3f} S {rS:.3f} diagS {rd:.3f}; H within 1e-12: {tight:.4f}")
    assert rH <= 1 and rS <= 1 and rd <= 1
    if method == "I":
        # full Hermitian S with a unit diagonal
        assert np.max(np.abs(S - S.conj().T)) == 0.0
        assert np.all(np.diag(S) == 1.0)
    else:
        rdH = _ratio(dH, o.diagH[:K], np.abs(o.diagH[:K]), np.diag(tolerance(pair_conditions(sysm, params))))
        assert rdH <= 1


def test_bordered_rows_match_full():
    """ComputeMatElem(Nmin, Nmax) with Nmin > 1 fills only the new rows and
    gives the same values as a full build."""
    sysm, params = synth.config_basis(1, K=100)
    with Context(sysm, 100) as a, Context(sysm, 100) as b:
        for c in (a, b):
            c.set_params(params)
        a.compute_mat_elem(1, 100, -1.1)
        b.compute_mat_elem(1, 70, -1.1)
        b.compute_mat_elem(71, 100, -1.1)
        Ha, Sa, dSa, _, _ = a.matrices(100)
        Hb, Sb, dSb, _, _ = b.matrices(100)
    lo = np.tril_indices(100)
    assert np.array_equal(Ha[lo], Hb[lo]) and np.array_equal(Sa, Sb) and np.array_equal(dSa, dSb)


@pytest.mark.parametrize("cfg,K,nfru", [(1, 90, 0), (1, 90, 60), (0, 120, 0)])
def test_deriv_matches_oracle(cfg, K, nfru):
    sysm, params = synth.config_basis(cfg, K=K)
    nfo = K - nfru
    lam = -0.55 if cfg == 0 else -1.1
    o = orc.Oracle(sysm, K, max_nfo=nfo)
    o.set_params(params)
    o.compute_mat_elem(1, nfru, lam) if nfru else None
    o.compute_mat_elem_and_deriv(nfru + 1, K, nfru, lam)
    with Context(sysm, K, max_nfo=nfo) as ctx:
        ctx.set_params(params)
        if nfru:
            ctx.compute_mat_elem(1, nfru, lam)
        ctx.compute_mat_elem_and_deriv(nfru + 1, K, nfru, lam)
        H, S, _, _, _ = ctx.matrices(K)
        D = ctx.deriv(nfo, K)
    Do = o.D[:, :nfo, :K]
    # only the entries StoreHSD writes: (i > nfru, j <= i) and their
    # conjugate partners (j > nfru)
    mask = np.zeros((nfo, K), dtype=bool)
    for i in range(nfru, K):
        mask[i - nfru, : i + 1] = True
        mask[i - nfru, i:] = True
    kap = pair_conditions(sysm, params)
    # derivative vectors apply C^-1 twice (F = C^-1 tCl M tCl C^-1 and the
    # Coulomb C^-1 J C^-1), so their rounding band is a few times wider
    tolD = tolerance(kap[nfru:, :], c=256.0)  # (nfo, K): pair (function, partner)
    # each derivative vector relative to its largest entry
    scale = np.max(np.abs(Do), axis=0)
    r = np.abs(D - Do).max(axis=0) / (np.where(scale > 0, scale, 1.0) * tolD)
    rD = float(np.max(r[mask]))
    lo = np.tril_indices(K)
    sH = np.abs(o.H[:K, :K][lo]) + abs(lam) * np.abs(o.S[:K, :K][lo])
    rH = _ratio(H[lo], o.H[:K, :K][lo], sH, tolerance(kap)[lo])
    print(f"cfg {cfg} nfru {nfru}: diff/tol D {rD:.3f} H {rH:.3f}")
    assert rD <= 1 and rH <= 1
