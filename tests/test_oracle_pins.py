"""Pins of the oracle where the reference ships no fixture (n = 3, 4,
several Y^+Y terms, derivatives):
* single pair terms against a 50-digit evaluation of the same formulas;
* its analytic EnergyIB gradient against central finite differences of its
  own energy (the reference's commented-out check, src/workproc.f90:4174-4203)."""
import numpy as np
import pytest

import mp_elements as mpe
import oracle as orc
from ecg_b200 import synth

EPS = np.finfo(float).eps


@pytest.mark.parametrize("name", ["h_minus_like", "h2_like", "li_like", "li_minus_like"])
def test_pair_terms_within_conditioning_of_50_digits(name):
    s = synth.make_system(name)
    b = synth.random_basis(s.n, 40, seed=7)
    o = orc.Oracle(s, 4)
    rng = np.random.default_rng(11)
    for _ in range(25):
        i, j, t = rng.integers(40), rng.integers(40), rng.integers(s.T)
        P = s.yhy_mats[t]
        h, sv, _, _ = o.matrix_elements(b[i], b[j], P, 0)
        hm, sm = mpe.term_energy(b[i], b[j], P, s.mass_matrix, s.charges)
        kap = mpe.term_condition(b[i], b[j], P)
        e = max(abs(h - hm) / max(abs(hm), abs(sm)), abs(sv - sm) / abs(sm))
        assert e <= 16 * EPS * kap + 1e-15


@pytest.mark.parametrize("cfg,K", [(1, 40), (0, 50)])
def test_oracle_gradient_matches_finite_differences(cfg, K):
    import scipy.linalg as sl
    sysm, params = synth.config_basis(cfg, K=K)
    o = orc.Oracle(sysm, K, max_nfo=K)
    o.set_params(params)
    o.compute_mat_elem(1, K, 0.0)
    H = np.tril(o.H[:K, :K]) + np.tril(o.H[:K, :K], -1).conj().T
    lam = sl.eigh(H, o.S[:K, :K], eigvals_only=True)[0] * (1 + 1e-10)
    o.last[:K] = 1.0
    E, g, err, _ = o.energy_ib(0, K, lam, 1e-12)
    rng = np.random.default_rng(2)
    for _ in range(6):
        f, m = int(rng.integers(K)), int(rng.integers(sysm.npt))
        h = 1e-6 * abs(params[f, m])
        es = []
        for sgn in (1, -1):
            p2 = params.copy()
            p2[f, m] += sgn * h
            o2 = orc.Oracle(sysm, K)
            o2.set_params(p2)
            o2.last[:K] = 1.0
            es.append(o2.energy_ia(1, K, lam, 1e-12, max_iter=40)[0])
        fd = (es[0] - es[1]) / (2 * h)
        o.activate()
        assert abs(fd - g[f * sysm.npt + m]) <= 1e-6 * np.max(np.abs(g)) + 1e-5 * abs(fd)
