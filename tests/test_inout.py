"""The reference's data file and swap file (ecg_b200.inout): the reader
against the known-answer fixtures, the writer against SaveResults' exact
text (src/workproc.f90:436-571), and the swap-file layout of
StoreMatricesInSwapFile / ReadSwapFileAndDistributeData
(src/workproc.f90:2158-2311) as a round trip through the oracle's matrices."""
import os

import numpy as np

import oracle as orc
from conftest import GOLDEN
from ecg_b200 import inout, synth

HERE = os.path.dirname(os.path.abspath(__file__))
TEXT = os.path.join(HERE, "golden", "inout_2_500.txt")


def test_read_matches_fixture(golden):
    f = inout.read_inout(TEXT)
    g = golden("inout_2_500")
    assert f.basis_size == g["K"] and f.which_eigenvalue == g["which"]
    assert f.current_energy == g["energy"] and f.invit_parameter == g["invit"] and f.eigval_tol == g["tol"]
    assert np.array_equal(f.masses, g["masses"]) and np.array_equal(f.charges, g["charges"])
    assert f.symmetry == g["symmetry"]
    assert np.array_equal(f.params, g["params"])
    assert len(f.history) == f.basis_size and len(f.bbop) == 10
    assert f.system().T == 1


def test_write_reproduces_saveresults(tmp_path):
    f = inout.read_inout(TEXT)
    out = tmp_path / "roundtrip.txt"
    inout.write_inout(f, out)
    assert out.read_text() == open(TEXT).read()


def test_fortran_d_format():
    assert inout.fortran_d(3670.4829652) == " 0.3670482965200000D+04"
    assert inout.fortran_d(-0.5891818196107302) == "-0.5891818196107302D+00"
    assert inout.fortran_d(1e-12) == " 0.1000000000000000D-11"
    assert inout.fortran_d(0.0) == " 0.0000000000000000D+00"


def test_swap_roundtrip(tmp_path):
    """pack -> file -> unpack gives back the layouts ReadSwapFile forms, for
    'I' (with a different lambda~ on the way back) and 'G'."""
    sysm, params = synth.config_basis(1, K=60)
    K = 60
    for method in ("I", "G"):
        o = orc.Oracle(sysm, K)
        o.set_params(params)
        lam1, lam2 = -1.05, -1.1
        o.compute_mat_elem(1, K, lam1, method=method)
        P = inout.pack_swap(o.H, o.S, o.diagH, method, lam1)
        path = tmp_path / f"swap_{method}.bin"
        inout.write_swap(path, P, o.diagS)
        assert inout.read_swap(path, K + 1) is None
        P2, dS = inout.read_swap(path, K)
        assert np.array_equal(P2, P) and np.array_equal(dS, o.diagS[:K])
        H, S, dH = inout.unpack_swap(P2, method, lam2)
        ref = orc.Oracle(sysm, K)
        ref.set_params(params)
        ref.compute_mat_elem(1, K, lam2, method=method)
        low = np.tril_indices(K, -1)
        scale = np.abs(ref.H[low]).max()
        assert np.max(np.abs(S[low] - ref.S[low])) == 0.0
        assert np.max(np.abs(H[low] - ref.H[low])) <= 1e-14 * scale
        if method == "I":
            assert np.max(np.abs(S - ref.S)) == 0.0
            assert np.max(np.abs(np.diag(H) - np.diag(ref.H))) <= 1e-14 * scale
        else:
            assert np.array_equal(dH, ref.diagH[:K])
