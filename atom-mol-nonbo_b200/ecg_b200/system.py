"""Physical system of one calculation: the inputs of the hot path that the
reference's ProgramDataInit derives from the input file
(src/workproc.f90:575-1202).

* mass matrix  M = 1/(2 m0) J + diag(1/(2 m_i))         (workproc.f90:606-610)
* pseudo-charges q0 (reference particle) and q_1..q_n   (workproc.f90:89-100)
* the Y^+Y symmetry projector as integer matrices acting on the nonlinear
  parameters, with integer coefficients               (workproc.f90:673-1202)

The Young-operator grammar is the reference's: factors in brackets, terms
joined by + or -, an optional integer coefficient, then products of pair
transpositions Pij of particles i, j (single digits), e.g. "(1+P12)(1+P34)".
"""
from collections import OrderedDict
import re

import numpy as np

__all__ = ["System", "transposition_matrix", "expand_y", "expand_yhy", "parse_young"]

_ALLOWED = set("0123456789P+-*()")


def transposition_matrix(p, q, npart):
    """Matrix of the pair transposition Pij on the n = npart-1 relative
    coordinates, as tabulated in src/workproc.f90:673-698.  P1i (i > 1) is the
    identity with column i-1 set to -1; Pij (i, j > 1) swaps coordinates i-1
    and j-1.  The table only fills P1i, not Pi1, so Pi1 is the identity
    there; this keeps that behaviour."""
    n = npart - 1
    m = np.eye(n, dtype=np.int64)
    if p == q:
        return m
    if not (1 <= p <= npart and 1 <= q <= npart):
        raise ValueError(f"transposition P{p}{q} outside 1..{npart}")
    if p == 1:
        m[:, q - 2] = -1
    elif q == 1:
        pass
    else:
        a, b = p - 2, q - 2
        m[a, a] = 0
        m[b, b] = 0
        m[b, a] = 1
        m[a, b] = 1
    return m


def parse_young(expr):
    """Split a Young-operator string into factors, each a list of
    (coefficient, [(p, q), ...]) terms, transpositions in written order."""
    s = expr.replace(" ", "").replace("*", "")
    bad = set(s) - _ALLOWED
    if bad:
        raise ValueError(f"Young operator contains invalid symbols: {sorted(bad)}")
    if s.count("(") != s.count(")"):
        raise ValueError("Young operator has unbalanced brackets")
    chunks, buf, i = [], "", 0
    while i < len(s):
        ch = s[i]
        if ch == "(":
            if buf:
                chunks.append(buf)
                buf = ""
            j = s.index(")", i)
            chunks.append(s[i + 1:j])
            i = j + 1
        else:
            buf += ch
            i += 1
    if buf:
        chunks.append(buf)
    factors = []
    for ch in chunks:
        if ch[0] not in "+-":
            ch = "+" + ch
        terms = []
        for sign, digits, perms in re.findall(r"([+-])(\d*)((?:P\d\d)*)", ch):
            if not digits and not perms:
                raise ValueError(f"empty term in factor {ch!r}")
            coef = int(sign + digits) if digits else (1 if sign == "+" else -1)
            terms.append((coef, [(int(t[1]), int(t[2])) for t in re.findall(r"P\d\d", perms)]))
        factors.append(terms)
    return factors


def _collect(terms):
    acc = OrderedDict()
    for c, m in terms:
        key = (m.shape, m.tobytes())
        if key in acc:
            acc[key][0] += c
        else:
            acc[key] = [c, m]
    return [(c, m) for c, m in acc.values() if c != 0]


def _factor_matrix(perms, npart, reverse=False):
    m = np.eye(npart - 1, dtype=np.int64)
    seq = perms if not reverse else perms[::-1]
    for p, q in seq:
        m = transposition_matrix(p, q, npart) @ m
    return m


def expand_y(expr, npart):
    """Expand Y itself into (coefficient, matrix) terms with identical
    matrices merged: Glob_YMatr / Glob_YCoeff (src/workproc.f90:920-1048),
    the last factor first, then right-multiplied by factors m-1 .. 1."""
    factors = parse_young(expr)
    terms = _collect([(c, _factor_matrix(pp, npart)) for c, pp in factors[-1]])
    for f in reversed(factors[:-1]):
        terms = _collect([(cs * ck, ms @ _factor_matrix(pk, npart)) for ck, pk in f for cs, ms in terms])
    return terms


def expand_yhy(expr, npart):
    """Expand Y^+Y into (coefficient, matrix) terms with identical matrices
    merged, in the order the reference produces them
    (src/workproc.f90:920-1202).  A product of permutation operators acts on
    the parameter matrices as the reversed product of their matrices."""
    factors = parse_young(expr)

    def mat(perms, reverse=False):
        return _factor_matrix(perms, npart, reverse)

    terms = expand_y(expr, npart)
    # Y^+Y: right-multiply by the reversed factors 1 .. m
    for f in factors:
        terms = _collect([(cs * ck, ms @ mat(pk, reverse=True)) for ck, pk in f for cs, ms in terms])
    return terms


class System:
    """Masses (m0 first), charges (q0 first) and the symmetry string."""

    def __init__(self, masses, charges, symmetry):
        self.masses = np.asarray(masses, dtype=np.float64)
        self.charges = np.asarray(charges, dtype=np.float64)
        if self.masses.shape != self.charges.shape or self.masses.size < 2:
            raise ValueError("masses and charges need one entry per particle")
        self.npart = self.masses.size
        self.n = self.npart - 1
        self.np = self.n * (self.n + 1) // 2
        self.npt = 2 * self.np
        self.symmetry = symmetry
        m = np.full((self.n, self.n), 0.5 / self.masses[0])
        m[np.diag_indices(self.n)] += 0.5 / self.masses[1:]
        self.mass_matrix = m
        terms = expand_yhy(symmetry, self.npart)
        self.yhy_coeffs = np.array([c for c, _ in terms], dtype=np.int32)
        self.yhy_mats = np.array([mm for _, mm in terms], dtype=np.int32)
        self.T = len(terms)
        yterms = expand_y(symmetry, self.npart)
        self.y_coeffs = np.array([c for c, _ in yterms], dtype=np.int32)
        self.y_mats = np.array([mm for _, mm in yterms], dtype=np.int32)

    @property
    def mass_matrix_cm(self):
        return np.asfortranarray(self.mass_matrix).ravel(order="F")

    @property
    def yhy_mats_cm(self):
        """Glob_YHYMatr(n, n, T) flattened column-major."""
        return np.ascontiguousarray(np.transpose(self.yhy_mats, (0, 2, 1))).ravel()

    @property
    def y_mats_cm(self):
        """Glob_YMatr(n, n, NumYTerms) flattened column-major."""
        return np.ascontiguousarray(np.transpose(self.y_mats, (0, 2, 1))).ravel()

    def __repr__(self):
        return f"System(n={self.n}, T={self.T}, symmetry={self.symmetry!r})"
