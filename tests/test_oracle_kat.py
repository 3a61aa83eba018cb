"""The oracle against the reference's own known answers: the six optimised
HD+ bases of example_input/ and the CURRENT_ENERGY stored with each (line 6
of each file).  lambda~ = CURRENT_ENERGY * INVITPARAMETER (src/main.f90:52)
selects WHICH_EIGENVALUE on the inverse-iteration path."""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle as orc
from conftest import FIXTURES
from ecg_b200 import System

TOL_E = 1e-10  # hartree


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_energy_matches_stored(golden, name):
    f = golden(name)
    sysm = System(f["masses"], f["charges"], f["symmetry"])
    assert sysm.T == 1
    K = f["K"]
    o = orc.Oracle(sysm, K)
    o.set_params(f["params"])
    o.last[:K] = 1.0
    E, err, it = o.energy_ia(1, K, f["energy"] * f["invit"], f["tol"])
    assert err in (0, 2)
    assert abs(E - f["energy"]) <= TOL_E


def test_oracle_g_path_matches_stored(golden):
    """The G path (ZHEGVX on the mirrored triangles, src/workproc.f90:1737-1750)
    on the K=500 bases, via SciPy's generalised Hermitian solver."""
    for name in ("inout_1_500", "inout_2_500"):
        f = golden(name)
        sysm = System(f["masses"], f["charges"], f["symmetry"])
        K = f["K"]
        o = orc.Oracle(sysm, K)
        o.set_params(f["params"])
        o.compute_mat_elem(1, K, 0.0, method="G")
        H = np.tril(o.H[:K, :K], -1)
        H = H + H.conj().T + np.diag(o.diagH[:K])
        S = np.tril(o.S[:K, :K], -1)
        S = S + S.conj().T + np.eye(K)
        w = f["which"]
        E = sl.eigh(H, S, eigvals_only=True, subset_by_index=[w - 1, w - 1])[0]
        assert abs(E - f["energy"]) <= 1e-9
