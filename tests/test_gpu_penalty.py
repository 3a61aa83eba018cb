"""The overlap penalty on the GPU (ecg_overlap_penalty: ComputeOverlapPenalty
and ComputeOverlapPenaltyAndAddGradient, src/workproc.f90:1491-1693) against
the oracle: the penalty value, and the gradient that mode 1 (the
reference's expression) and mode 2 (the derivative of the penalty) add to
the context's gradient after the fused adjoint EnergyGB, with the Glob_D
derivatives the reference reads recomputed on the GPU for the flagged pairs
and taken from the oracle's ComputeMatElemAndDeriv there."""
import numpy as np
import pytest

import oracle as orc
from ecg_b200 import Context, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg,K,nfru,t2", [(1, 60, 0, 0.02), (1, 60, 20, 0.3), (0, 80, 10, 0.05),
                                          (4, 40, 5, 0.1)])
def test_penalty_against_oracle(cfg, K, nfru, t2):
    b = 0.7
    sysm, params = synth.config_basis(cfg, K=K)
    npt = sysm.npt
    o = orc.Oracle(sysm, K, max_nfo=K)
    o.set_params(params)
    o.compute_mat_elem(1, max(nfru, 1), 0.0, method="G")
    o.compute_mat_elem_and_deriv(nfru + 1, K, nfru, 0.0, method="G")
    tp_o = o.overlap_penalty(nfru, K, b, t2)
    g1_o = np.zeros((K - nfru) * npt)
    g2_o = np.zeros((K - nfru) * npt)
    o.overlap_penalty(nfru, K, b, t2, g1_o)
    o.overlap_penalty(nfru, K, b, t2, g2_o, exact=True)
    with Context(sysm, K, method="G") as ctx:
        ctx.set_params(params)
        ctx.compute_mat_elem(1, K, 0.0)   # rows 1..nfru, as earlier steps leave them in the reference
        E, g0, err = ctx.energy_gb_adjoint(nfru, K, which=1)
        assert err == 0
        tp0, _ = ctx.overlap_penalty(nfru, K, b, t2, mode=0)
        tp1, g1 = ctx.overlap_penalty(nfru, K, b, t2, mode=1)
        tp2, g2 = ctx.overlap_penalty(nfru, K, b, t2, mode=2)
    flagged = np.sum(np.abs(np.tril(o.S[:K, :K], -1)) ** 2 > t2)
    d1 = g1 - g0          # mode 1 added to the EnergyGB gradient
    d2 = g2 - g1          # mode 2 added on top of that
    scale = max(np.max(np.abs(g1_o)), 1e-300)
    e1 = np.max(np.abs(d1 - g1_o)) / scale
    e2 = np.max(np.abs(d2 - g2_o)) / max(np.max(np.abs(g2_o)), 1e-300)
    rnd = 1e-14 * max(np.max(np.abs(g0)), np.max(np.abs(g1))) / scale  # rounding of the differences
    print(f"cfg {cfg} K={K} nfru={nfru} t2={t2}: {flagged} flagged pairs, penalty {tp0:.12g} (oracle {tp_o:.12g}), "
          f"gradient rel diff mode 1 {e1:.1e}, mode 2 {e2:.1e}")
    assert flagged > 0
    assert tp0 == tp1 == tp2
    assert abs(tp0 - tp_o) <= 1e-12 * tp_o
    assert e1 <= 1e-9 + rnd
    assert e2 <= 1e-9 + rnd


def test_penalty_nothing_flagged():
    """A threshold above every overlap: zero penalty and the gradient unchanged."""
    sysm, params = synth.config_basis(1, K=30)
    with Context(sysm, 30, method="G") as ctx:
        ctx.set_params(params)
        E, g0, err = ctx.energy_gb_adjoint(0, 30, which=1)
        tp, g = ctx.overlap_penalty(0, 30, 0.7, 0.999999, mode=1)
    assert tp == 0.0
    assert np.array_equal(g, g0)
