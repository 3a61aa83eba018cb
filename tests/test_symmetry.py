"""Y^+Y expansion (the outputs of src/workproc.f90:673-1202 that the hot
path consumes), checked against an independent group-algebra expansion."""
import itertools
from collections import defaultdict

import numpy as np
import pytest

from ecg_b200 import System, expand_yhy, parse_young, transposition_matrix


def test_transposition_tables():
    # P1i: identity with column i-1 = -1 (src/workproc.f90:686-688)
    np.testing.assert_array_equal(transposition_matrix(1, 3, 4), [[1, -1, 0], [0, -1, 0], [0, -1, 1]])
    # Pij swaps coordinates i-1, j-1 (src/workproc.f90:689-698)
    np.testing.assert_array_equal(transposition_matrix(3, 4, 4), [[1, 0, 0], [0, 0, 1], [0, 1, 0]])
    np.testing.assert_array_equal(transposition_matrix(4, 3, 4), transposition_matrix(3, 4, 4))
    np.testing.assert_array_equal(transposition_matrix(1, 1, 4), np.eye(3))


def test_parse():
    f = parse_young("(1+P12)(1 - P34) * 2P23")
    assert f == [[(1, []), (1, [(1, 2)])], [(1, []), (-1, [(3, 4)])], [(2, [(2, 3)])]]
    with pytest.raises(ValueError):
        parse_young("(1+Q12)")
    with pytest.raises(ValueError):
        parse_young("(1+P12")


def _perm_of(p, q, npart):
    s = list(range(npart))
    s[p - 1], s[q - 1] = s[q - 1], s[p - 1]
    return tuple(s)


def _compose(a, b):  # (a b)(x) = a(b(x))
    return tuple(a[b[i]] for i in range(len(a)))


def _coord_matrix(perm, npart):
    """Matrix of a particle permutation on the relative coordinates
    r_i - r_1 (i = 2..npart) built directly from its action."""
    n = npart - 1
    M = np.zeros((n, n), dtype=np.int64)
    # new coordinate i: r_{perm(i+1)} - r_{perm(0)}
    for i in range(n):
        a, b = perm[i + 1], perm[0]
        if a != 0:
            M[i, a - 1] += 1
        if b != 0:
            M[i, b - 1] -= 1
    return M


@pytest.mark.parametrize("expr,npart", [("(1+P23)", 3), ("(1+P12)(1+P34)", 4), ("(1+P23)(1-P24)", 4),
                                        ("(1+P23)(1+P45)(1-P24)", 5), ("(1-P12)", 3), ("(P11)", 3)])
def test_expansion_matches_group_algebra(expr, npart):
    # Y^+Y in the group algebra; Y^+ reverses factor and product order and
    # transpositions are involutions.
    factors = parse_young(expr)
    ident = tuple(range(npart))

    def elem(perms):
        g = ident
        for p, q in perms:
            g = _compose(g, _perm_of(p, q, npart))
        return g

    Y = {ident: 1}
    for f in factors:
        new = defaultdict(int)
        for g, c in Y.items():
            for ck, pk in f:
                new[_compose(g, elem(pk))] += c * ck
        Y = dict(new)
    YH = {tuple(np.argsort(g)): c for g, c in Y.items()}  # inverses
    YHY = defaultdict(int)
    for a, ca in YH.items():
        for b, cb in Y.items():
            YHY[_compose(a, b)] += ca * cb
    # expected (matrix, coefficient) multiset; mapping group elements to
    # matrices through the transposition tables (only P1i and Pij with
    # i, j > 1 occur in these strings)
    exp = defaultdict(int)
    for g, c in YHY.items():
        if c:
            exp[_coord_matrix(g, npart).tobytes()] += c
    exp = {k: v for k, v in exp.items() if v}
    got = {m.astype(np.int64).tobytes(): c for c, m in expand_yhy(expr, npart)}
    # the coordinate representation is a homomorphism or anti-homomorphism;
    # compare the multiset of coefficients and the set of matrices up to
    # transposition of every matrix
    assert sorted(exp.values()) == sorted(got.values())
    n = npart - 1
    exp_m = {np.frombuffer(k, dtype=np.int64).reshape(n, n).tobytes() for k in exp}
    got_m = {np.frombuffer(k, dtype=np.int64).reshape(n, n).tobytes() for k in got}
    got_t = {np.frombuffer(k, dtype=np.int64).reshape(n, n).T.copy().tobytes() for k in got}
    assert exp_m == got_m or exp_m == got_t


def test_config_systems():
    s = System([1836.15, 1.0, 1.0], [1.0, -1.0, -1.0], "(1+P23)")
    assert s.T == 2 and list(s.yhy_coeffs) == [2, 2]
    s = System([1836.15, 1836.15, 1.0, 1.0], [1.0, 1.0, -1.0, -1.0], "(1+P12)(1+P34)")
    assert s.T == 4 and list(s.yhy_coeffs) == [4, 4, 4, 4]
    s = System([12786.0, 1.0, 1.0, 1.0], [3.0, -1.0, -1.0, -1.0], "(1+P23)(1-P24)")
    assert s.T == 6
    # mass matrix (src/workproc.f90:606-610)
    m = s.mass_matrix
    assert np.allclose(m, 0.5 / 12786.0 + np.diag([0.5, 0.5, 0.5]))
