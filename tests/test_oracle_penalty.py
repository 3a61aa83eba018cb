"""The oracle's overlap penalty (ComputeOverlapPenalty /
ComputeOverlapPenaltyAndAddGradient, src/workproc.f90:1491-1693): the
penalty against a direct sum over the normalised overlaps; the gradient in
the derivative mode against central differences of the penalty; and the
reference's own gradient expression, which is not that derivative (its
normalisation terms carry sqrt(diagS_i/diagS_j), and the lower-index
function gets S_ji^2 where the derivative has |S_ji|^2), against an
independent restatement of that expression from Glob_D."""
import numpy as np

import oracle as orc
from ecg_b200 import synth

K, NFRU, B, T2 = 12, 4, 0.7, 0.02


def setup():
    sysm, params = synth.config_basis(1, K=K)
    o = orc.Oracle(sysm, K, max_nfo=K)
    return sysm, params, o


def prep(o, params, deriv):
    o.set_params(params)
    o.compute_mat_elem(1, NFRU, 0.0, method="G")
    if deriv:
        o.compute_mat_elem_and_deriv(NFRU + 1, K, NFRU, 0.0, method="G")
    else:
        o.compute_mat_elem(NFRU + 1, K, 0.0, method="G")


def test_penalty_value():
    sysm, params, o = setup()
    prep(o, params, False)
    S = o.S[:K, :K]
    pc = B / (1 - T2)
    want = sum(pc * (abs(S[j, i]) ** 2 - T2) for i in range(K) for j in range(max(i + 1, NFRU), K)
               if abs(S[j, i]) ** 2 > T2)
    got = o.overlap_penalty(NFRU, K, B, T2)
    assert want > 0
    assert abs(got - want) <= 1e-14 * want


def test_penalty_gradient_modes():
    sysm, params, o = setup()
    npt = sysm.npt
    prep(o, params, True)
    g_ref = np.zeros((K - NFRU) * npt)
    g_ex = np.zeros((K - NFRU) * npt)
    o.overlap_penalty(NFRU, K, B, T2, g_ref)
    o.overlap_penalty(NFRU, K, B, T2, g_ex, exact=True)
    # the reference's expression restated from Glob_D
    S, D, dS = o.S, o.D, o.diagS
    pc = B / (1 - T2)
    g_py = np.zeros_like(g_ref)
    for i in range(1, K + 1):
        for j in range(max(i + 1, NFRU + 1), K + 1):
            s = S[j - 1, i - 1]
            if abs(s) ** 2 <= T2:
                continue
            t = np.sqrt(dS[i - 1] / dS[j - 1])
            for m in range(npt):
                g_py[(j - NFRU - 1) * npt + m] += 2 * pc * (s * np.conj(
                    D[npt + m, j - NFRU - 1, i - 1] - 0.5 * D[npt + m, j - NFRU - 1, j - 1] * s * t)).real
                if i > NFRU:
                    g_py[(i - NFRU - 1) * npt + m] += 2 * pc * (s * (
                        D[npt + m, i - NFRU - 1, j - 1] - 0.5 * D[npt + m, i - NFRU - 1, i - 1] * s / t)).real
    assert np.max(np.abs(g_ref - g_py)) <= 1e-13 * np.max(np.abs(g_py))
    # central differences of the penalty
    fd = np.zeros_like(g_ref)
    for r in range(NFRU, K):
        for m in range(npt):
            pp = params.copy()
            h = 1e-6 * max(1.0, abs(pp[r, m]))
            pp[r, m] += h
            prep(o, pp, False)
            a = o.overlap_penalty(NFRU, K, B, T2)
            pp[r, m] -= 2 * h
            prep(o, pp, False)
            b = o.overlap_penalty(NFRU, K, B, T2)
            fd[(r - NFRU) * npt + m] = (a - b) / (2 * h)
    scale = np.max(np.abs(fd))
    dev_ex = np.max(np.abs(g_ex - fd)) / scale
    dev_ref = np.max(np.abs(g_ref - fd)) / scale
    print(f"derivative mode vs central differences: {dev_ex:.1e}; reference expression: {dev_ref:.1e}")
    assert dev_ex <= 1e-6
