"""The C ABI library loads and exports every function include/ecg_abi.h
declares (no GPU work is issued: loading does not touch the device)."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "ecg_abi.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ecg_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared()
    for must in ("ecg_ctx_create", "ecg_compute_mat_elem", "ecg_compute_mat_elem_and_deriv", "ecg_ghepiis",
                 "ecg_energy_ia", "ecg_energy_ib", "ecg_energy_ib_adjoint", "ecg_matrix_elements"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from ecg_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers exactly the declared set
    assert sorted(_lib.PROTOTYPES) == declared()


def test_binding_fails_loudly_without_library(tmp_path, monkeypatch):
    from ecg_b200 import _lib
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    import pytest
    with pytest.raises(OSError):
        _lib.load()
