"""Expectation values over an eigenvector: the result layout of
ExpectationValuesG (src/workproc.f90:7785-8600) and its printed block.

`ecg_expectation_values` returns the 6 np + 9 sums in the reference's MEkl
order (src/workproc.f90:8045-8060); `unpack` turns them into named values,
the pair quantities as symmetric n x n matrices (row/column a = coordinate
r_a, off-diagonal (a, b) = r_ab), each with its error bound under the
name + "_e".  `report_lines` formats the scalar block the reference prints
(src/workproc.f90:8432-8452)."""
import numpy as np

from .inout import fortran_d

__all__ = ["PAIR_NAMES", "SCALAR_NAMES", "FINE_STRUCTURE", "unpack", "report_lines"]

PAIR_NAMES = ("rm2", "rm", "r", "r2", "deltar", "drach_deltar")
SCALAR_NAMES = ("H", "S", "T", "V", "MV", "drach_MV", "Darwin", "drach_Darwin", "OO")
FINE_STRUCTURE = 7.2973525376e-03  # Glob_FineStructConst, CODATA 2006 (src/globvars.f90:37)


def unpack(values, errors, n):
    """Named expectation values from the MEkl-ordered sums."""
    np_ = n * (n + 1) // 2
    out = {}
    for b, name in enumerate(PAIR_NAMES):
        for suffix, src in (("", values), ("_e", errors)):
            m = np.zeros((n, n))
            c = b * np_
            for a in range(n):
                for bb in range(a, n):
                    m[a, bb] = m[bb, a] = src[c]
                    c += 1
            out[name + suffix] = m
    for k, name in enumerate(SCALAR_NAMES):
        out[name] = float(values[6 * np_ + k])
        out[name + "_e"] = float(errors[6 * np_ + k])
    return out


def report_lines(d):
    """The scalar lines of the reference's report, value then the relative
    error estimate |X_e / X|, in its (2x,a23,d23.16,a3,d12.5,a1) format."""
    a2 = FINE_STRUCTURE ** 2
    rows = [("H", d["H"], "H"), ("S", d["S"], "S"), ("T", d["T"], "T"), ("V", d["V"], "V"),
            ("MV", d["MV"], "MV"), ("drach_MV", d["drach_MV"], "drach_MV"),
            ("8*MV", 8 * d["MV"], "MV"), ("8*drach_MV", 8 * d["drach_MV"], "drach_MV"),
            ("Darwin", d["Darwin"], "Darwin"), ("drach_Darwin", d["drach_Darwin"], "drach_Darwin"),
            ("OO", d["OO"], "OO"),
            ("(alpha^2)*MV", d["MV"] * a2, "MV"), ("(alpha^2)*drach_MV", d["drach_MV"] * a2, "drach_MV"),
            ("(alpha^2)*Darwin", d["Darwin"] * a2, "Darwin"),
            ("(alpha^2)*drach_Darwin", d["drach_Darwin"] * a2, "drach_Darwin"),
            ("(alpha^2)*OO", d["OO"] * a2, "OO")]
    lines = []
    for label, v, base in rows:
        rel = abs(d[base + "_e"] / d[base]) if d[base] != 0 else float("inf")
        lines.append("  " + (label + "=").rjust(23) + fortran_d(v) + "  (" + fortran_d(rel, 12, 5) + ")")
    return lines
