"""Algorithmic operation counts of one pair term, for the roofline.

Walks the loop nests of the reference's MatrixElements
(src/matelem.f90:109-748, as restated in ecg_oracle.c) and of the adjoint
reformulation (ecg_grad.cuh, term_adjoint) and tallies FP64 operations
with these rules: complex multiply 6, complex add/sub 2, real x complex 2,
real multiply or add 1; complex divide, reciprocal and square root counted
as one operation each and reported separately ("div", "sqrt").

TEST/BENCH INFRASTRUCTURE: bench.py reads these counts; nothing in the
product imports this module.
"""


class Tally:
    def __init__(self):
        self.flop = 0
        self.div = 0
        self.sqrt = 0

    def total(self):
        return self.flop + self.div + self.sqrt

    def as_dict(self):
        return {"flop": self.flop, "div": self.div, "sqrt": self.sqrt, "total": self.total()}


CMUL, CADD, RC, CMAC = 6, 2, 2, 8


def _energy(n, t, coulomb_cube=True):
    np_ = n * (n + 1) // 2
    # A = L L' for bra and ket (sum k = 1..j)
    t.flop += 2 * sum(2 * (j + 1) for i in range(n) for j in range(i, n))
    # P'AP and P'BP: W (n^2 x n, two sums) and the symmetric result
    t.flop += 4 * n ** 3 + 4 * n * np_
    t.flop += 2 * n                      # det L_k, det L_l
    t.flop += CADD * np_                 # C = Ck + tCl
    for i in range(n):                   # pseudo-Cholesky
        for j in range(i, n):
            t.flop += CMAC * i
            if i == j:
                t.sqrt += 1
                t.flop += CMUL           # det
            else:
                t.div += 1
    for i in range(n):                   # invert the factor
        t.div += 1
        for j in range(i + 1, n):
            t.flop += CMAC * (j - i)
            t.div += 1
    t.flop += sum(CMAC * (n - j) for i in range(n) for j in range(i, n))  # inv = X'X
    t.flop += 1 + 2 + CMUL               # S = 2^(3n/2) c sqrt(c)
    t.div += 1
    t.sqrt += 1
    t.flop += 2 * CMAC * n ** 3 + 4 * n * n + 2 + CMUL   # T
    t.flop += 2                          # cnumb
    npairs = n * (n - 1) // 2
    # V: per diagonal i and per pair i<j
    t.flop += n * (2 * 1 + 2 + 2) + 2 + npairs * (3 * CADD + 1 + 2 + 2)
    t.div += n + npairs
    t.sqrt += n + npairs
    if coulomb_cube:                     # tr[C^-1 J]^(-3/2) kept for the gradient
        t.flop += (n + npairs) * CMUL
        t.div += n + npairs
    t.flop += CADD                       # H = T + V


def reference_term(n, gradflag):
    """Counts of one MatrixElements call (the reference computes the
    Coulomb cubes even without gradient)."""
    t = Tally()
    _energy(n, t)
    np_ = n * (n + 1) // 2
    gk = gradflag in (1, 3)
    gl = gradflag in (2, 3)
    tri = sum(n - j for j in range(n))               # lower-triangular product, per row
    inv_l = sum(2 * (j - i) + 1 for i in range(n) for j in range(i + 1, n))  # real L^-1
    for side in (gk, gl):
        if not side:
            continue
        t.flop += RC * n * tri                       # inv * L (lower)
        t.flop += inv_l
        t.div += n                                   # 1/L_ii
        t.flop += 2 + np_ * (2 + CMUL) + CMUL + CMUL + np_ * CMUL   # dS/dL, dS/dB
    if gl:
        t.flop += 2 * (2 * n ** 3)                   # P inv P' (real x complex sums)
    for side in (gl, gk):                            # dT: X = C^-1 Y M Y C^-1, then X L
        if not side:
            continue
        t.flop += RC * n ** 3 + CMAC * n ** 3 + CMAC * n ** 3 + CMAC * n * np_
        t.flop += RC * n * tri + 2 * np_ * (CMUL + CMUL + CADD) + CMUL * 2
        t.div += 1                                   # T/S
    if gl:
        t.flop += 2 * (2 * n ** 3)                   # G = P X P'
    npair = n * (n + 1) // 2
    # dV: per (i, j<=i) the matrix tQ, then tQ L (and P tQ P', ttQ L)
    per = n * n * 4 * CMUL // 2 + CMAC * np_
    for side in (gk, gl):
        if side:
            t.flop += npair * (per + RC * tri * n + np_ * 2 * (CMAC + 2))
    if gl:
        t.flop += npair * 4 * n ** 3
    t.flop += (gk + gl) * np_ * 2 * (CMAC + CMAC)  # final combination
    t.div += (gk + gl) * 1                         # V/S
    return t


def adjoint_term(n, ket=True):
    """Counts of one term of the adjoint pass: the energy part (without the
    Coulomb cubes of the reference), the Coulomb weights, the two middle
    matrices and sandwiches, the permutation of the ket side and the
    coefficient accumulation."""
    t = Tally()
    _energy(n, t, coulomb_cube=False)
    np_ = n * (n + 1) // 2
    npairs = n * (n + 1) // 2
    t.flop += npairs * (CMUL + 3 * CADD) + 3     # weights (the a + a - 2b traces, products)
    t.div += npairs
    t.sqrt += npairs
    t.flop += CMUL + 2 * 2                        # a = 1.5 (H - E S)
    t.flop += n * (n - 1) * CADD + np_ * CMUL + 2  # Q scaled
    sides = 2 if ket else 1
    # middle R = 6 S Y M Y + Qs, sandwich inv R inv, Z = a inv - X, accumulate
    t.flop += sides * (RC * n ** 3 + CMAC * n * np_ + CMUL + CADD * np_)
    t.flop += sides * (CMAC * n ** 3 + CMAC * n * np_)
    t.flop += sides * np_ * (CMUL + CADD + RC + CADD)
    if ket:
        t.flop += 2 * n ** 3 + 2 * n * np_        # P Z P'
    return t


def pair_counts(n, T):
    """Per pair (sum over T terms): reference energy-only, reference with
    gradflag 3, adjoint."""
    return {
        "reference_energy": {k: v * T for k, v in reference_term(n, 0).as_dict().items()},
        "reference_grad3": {k: v * T for k, v in reference_term(n, 3).as_dict().items()},
        "adjoint": {k: v * T for k, v in adjoint_term(n).as_dict().items()},
    }


if __name__ == "__main__":
    import json
    for n in (2, 3, 4, 5):
        print(n, json.dumps({"energy": reference_term(n, 0).as_dict(), "grad3": reference_term(n, 3).as_dict(),
                             "adjoint": adjoint_term(n).as_dict()}))
