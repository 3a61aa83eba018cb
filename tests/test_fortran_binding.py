"""The iso_c_binding interfaces of the Fortran host module
(atom-mol-nonbo_b200/fortran/ecg_gpu.f90) against the C declarations in
include/ecg_abi.h: every bind(C) name exists, with the same number of
arguments, and each argument has the matching Fortran kind and passing
(value for C scalars; by reference for C pointers, intent(in) where the C
pointer is const).  No Fortran compiler is needed: both files are parsed as
text."""
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "ecg_abi.h")
F90 = os.path.join(ROOT, "atom-mol-nonbo_b200", "fortran", "ecg_gpu.f90")


def c_decls():
    txt = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(int|long long)\s+(ecg_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", txt, flags=re.S):
        args = [a.strip() for a in m.group(3).replace("\n", " ").split(",") if a.strip() and a.strip() != "void"]
        parsed = []
        for a in args:
            mm = re.match(r"^(const\s+)?([A-Za-z_ ]+?)\s*(\**)\s*([A-Za-z_][A-Za-z0-9_]*)$", a)
            assert mm, a
            parsed.append({"const": bool(mm.group(1)), "base": mm.group(2).strip(), "ptr": len(mm.group(3)),
                           "name": mm.group(4)})
        out[m.group(2)] = {"ret": m.group(1), "args": parsed}
    return out


def f_interfaces():
    txt = open(F90).read()
    body = txt[txt.index("interface"):txt.index("end interface")]
    # join continuation lines
    body = re.sub(r"&\s*\n\s*", " ", body)
    out = {}
    for m in re.finditer(r"integer\(c_int\)\s+function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name='(\w+)'\)(.*?)end function",
                         body, flags=re.S):
        args = [a.strip() for a in m.group(2).split(",") if a.strip()]
        decl = {}
        for line in m.group(4).splitlines():
            line = line.strip()
            if "::" not in line or line.startswith("import"):
                continue
            spec, names = line.split("::")
            spec = spec.replace(" ", "").lower()
            for nm in re.findall(r"(\w+)(\(\*\))?", names):
                decl[nm[0]] = {"spec": spec, "array": bool(nm[1])}
        out[m.group(3)] = {"fname": m.group(1), "args": [(a, decl.get(a)) for a in args]}
    return out


def _expect(carg):
    """(allowed Fortran type prefixes, by value?) for one C argument."""
    base, ptr = carg["base"], carg["ptr"]
    if base == "ecg_ctx":
        return (["type(c_ptr)"], ptr == 1)
    if base == "void" and ptr == 1:
        return (["type(c_ptr)"], True)
    if ptr == 0:
        return ({"int": ["integer(c_int)"], "double": ["real(c_double)"], "char": ["character(kind=c_char)"]}[base],
                True)
    # complex Fortran arrays travel as (re, im) double pairs
    return ({"int": ["integer(c_int)"], "double": ["real(c_double)", "complex(c_double_complex)"]}[base], False)


def test_every_interface_matches_the_header():
    cd = c_decls()
    fi = f_interfaces()
    assert len(fi) >= 10
    for cname, f in fi.items():
        assert cname in cd, f"{cname} is bound in ecg_gpu.f90 but not declared in ecg_abi.h"
        assert f["fname"] == cname, (f["fname"], cname)
        cargs = cd[cname]["args"]
        assert len(f["args"]) == len(cargs), (cname, [a for a, _ in f["args"]], [a["name"] for a in cargs])
        for (fa, d), ca in zip(f["args"], cargs):
            assert d is not None, f"{cname}: argument {fa} has no declaration"
            types, by_value = _expect(ca)
            assert any(d["spec"].startswith(t) for t in types), (cname, fa, d["spec"], ca)
            assert (",value" in d["spec"]) == by_value, (cname, fa, d["spec"], ca)
            if ca["ptr"] and ca["const"]:
                assert "intent(in)" in d["spec"], (cname, fa, d["spec"])
            if ca["ptr"] and not ca["const"] and ca["base"] not in ("ecg_ctx", "void"):
                assert "intent(out)" in d["spec"] or "intent(inout)" in d["spec"], (cname, fa, d["spec"])


def test_parser_sees_the_main_entry_points():
    fi = f_interfaces()
    for must in ("ecg_ctx_create", "ecg_compute_mat_elem", "ecg_ghepiis", "ecg_energy_ia", "ecg_energy_ib_adjoint",
                 "ecg_eval_candidates", "ecg_eval_candidates_grad"):
        assert must in fi, must


@pytest.mark.parametrize("bad", ["value_to_ref", "drop_arg"])
def test_checker_catches_a_drift(bad, monkeypatch, tmp_path):
    """A planted mismatch in a copy of the Fortran file is reported."""
    orig = txt = open(F90).read()
    if bad == "value_to_ref":
        txt = txt.replace("integer(c_int), value :: nmin, nmax\n    real(c_double), value :: approx_energy",
                          "integer(c_int), intent(in) :: nmin, nmax\n    real(c_double), value :: approx_energy", 1)
    else:
        txt = txt.replace("function ecg_compute_mat_elem(ctx, nmin, nmax, approx_energy)",
                          "function ecg_compute_mat_elem(ctx, nmin, approx_energy)", 1)
    assert txt != orig
    p = tmp_path / "ecg_gpu.f90"
    p.write_text(txt)
    monkeypatch.setattr(__import__(__name__), "F90", str(p))
    with pytest.raises(AssertionError):
        test_every_interface_matches_the_header()
