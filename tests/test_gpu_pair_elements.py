"""MatrixElements (src/matelem.f90:12-750) on the GPU against the oracle:
one call per (bra, ket, permutation) triple, every gradflag, n = 2, 3, 4."""
import numpy as np
import pytest

import oracle as orc
from ecg_b200 import Context, synth
from gpu_util import term_conditions, tolerance

pytestmark = pytest.mark.gpu

# Per call: H relative to max(|H|, |S|), S relative to |S|, each derivative
# vector relative to its largest entry; allowed: 1e-12, or 64 eps cond(C)
# for terms whose C is ill-conditioned (the oracle itself is within
# 4 eps cond(C) of 50-digit values, tests/test_oracle_pins.py).


@pytest.mark.parametrize("name", ["h_minus_like", "h2_like", "li_like", "li_minus_like"])
@pytest.mark.parametrize("gradflag", [0, 1, 2, 3])
def test_matrix_elements_match_oracle(name, gradflag):
    sysm = synth.make_system(name)
    basis = synth.random_basis(sysm.n, 64, seed=7)
    rng = np.random.default_rng(11)
    cnt = 256
    ik = rng.integers(0, 64, cnt)
    il = rng.integers(0, 64, cnt)
    il[:8] = ik[:8]  # include k == l
    terms = rng.integers(0, sysm.T, cnt).astype(np.int32)
    pk, pl = basis[ik], basis[il]
    o = orc.Oracle(sysm, 4)
    with Context(sysm, 4) as ctx:
        H, S, Dk, Dl = ctx.matrix_elements(pk, pl, terms, gradflag)
    kap = term_conditions(sysm, pk, pl, terms)
    # derivative vectors apply C^-1 twice, so their band is wider
    tol = tolerance(kap, c=256.0 if gradflag else 64.0)
    worst, worst_ratio, n_tight = 0.0, 0.0, 0
    for i in range(cnt):
        h, s, dk, dl = o.matrix_elements(pk[i], pl[i], sysm.yhy_mats[terms[i]], gradflag)
        e = max(abs(H[i] - h) / max(abs(h), abs(s)), abs(S[i] - s) / abs(s))
        if gradflag in (1, 3):
            e = max(e, np.max(np.abs(Dk[i] - dk)) / np.max(np.abs(dk)))
        if gradflag in (2, 3):
            e = max(e, np.max(np.abs(Dl[i] - dl)) / np.max(np.abs(dl)))
        worst = max(worst, e)
        worst_ratio = max(worst_ratio, e / tol[i])
        n_tight += e <= 1e-12
    print(f"{name} gradflag={gradflag}: worst rel diff {worst:.2e}, {n_tight}/{cnt} within 1e-12, "
          f"worst diff/tolerance {worst_ratio:.3f}")
    assert worst_ratio <= 1.0


def test_unit_overlap_identity():
    """S_kk = 1 for P = identity (the 2^(3n/2) normalisation,
    src/matelem.f90:244-245)."""
    sysm = synth.make_system("h2_like")
    basis = synth.random_basis(sysm.n, 100, seed=3)
    t0 = np.zeros(100, dtype=np.int32)
    with Context(sysm, 4) as ctx:
        _, S, _, _ = ctx.matrix_elements(basis, basis, t0, 0)
    assert np.all(np.abs(S - 1.0) <= tolerance(term_conditions(sysm, basis, basis, t0)))
