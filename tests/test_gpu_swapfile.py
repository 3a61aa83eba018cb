"""Resuming a GPU context from the reference's swap file (ecg_set_matrices,
ReadSwapFileAndDistributeData, src/workproc.f90:2158-2240): H and S stored by
one context with one lambda~ and read back into a fresh context with
another give the energy of a full recomputation, on the 'I' path
(EnergyIA with AreMatElemNeeded = .false.) and the 'G' path (EnergyGA)."""
import numpy as np
import pytest

from ecg_b200 import Context, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method", ["I", "G"])
def test_resume_from_swap_file(tmp_path, method):
    sysm, params = synth.config_basis(1, K=300)
    K = 300
    path = str(tmp_path / "swap.bin")
    lam1 = -1.0
    with Context(sysm, K, method=method) as a:
        a.set_params(params)
        a.compute_mat_elem(1, K, lam1)
        a.store_swap(path, K, lam1)
        if method == "I":
            a.set_vectors(K, last_eigvec=np.ones(K, dtype=np.complex128))
            E0, _, _ = a.energy_ia(1, K, -1.2, -1e-12, max_iter=100)
            lam2 = E0 * 1.000001
            a.set_vectors(K, last_eigvec=np.ones(K, dtype=np.complex128))
            Eref, erra, _ = a.energy_ia(1, K, lam2, 1e-12)
        else:
            Eref, erra, _ = a.energy_ga(1, K, which=1)
    with Context(sysm, K, method=method) as b:
        b.set_params(params)
        assert not b.read_swap(path, K + 1) if K + 1 <= b.ld else True
        if method == "I":
            assert b.read_swap(path, K, lam2)
            b.set_vectors(K, last_eigvec=np.ones(K, dtype=np.complex128))
            E, err, _ = b.energy_ia(1, K, lam2, 1e-12, mat_elem_needed=False)
        else:
            assert b.read_swap(path, K)
            E, err, _ = b.energy_ga(1, K, which=1, mat_elem_needed=False)
    print(f"{method}: recomputed E={Eref:.15f} resumed E={E:.15f} diff {E - Eref:.1e}")
    assert err == erra == 0
    assert abs(E - Eref) <= 1e-12
