"""Analytic far-field multipole tables (index_cc, cc, n_cc_lm_ijk, index_ijk_max_cc).

The reference's far-field sum-up (fast_rap_src_dfpt_gpu_eval/sum_up_whole_potential.cpp:91-187)
evaluates, per (point, atom) pair,

    dpot = sum_{n < n_cc_lm_ijk[l_max]}  x^i y^j z^k * Fp[nn] * cc[n] * Q[l(n), m(n)]

with (l, m, i, j, k, nn) = index_cc[n, 0:6], Fp[0] = 1/r and
Fp[n] = Fp[n-1] * (1 - 2n) / r^2, i.e. Fp[n] = (-1)^n (2n-1)!! / r^(2n+1).
The tables come from the host application (FHI-aims) and are not in the
reference repository, so this module derives them from the mathematics:

    sum_lm Q_lm r^-(l+1) Y_lm(r_hat) = sum_lm Q_lm R_lm(x, y, z) / r^(2l+1)

where R_lm = r^l Y_lm is the regular solid harmonic in the reference's real
Y_lm convention (fast_rap_src_dfpt_gpu_eval/sheval.hpp:6-343).  Every x^2 in
R_lm is replaced by r^2 - y^2 - z^2 until x appears at most linearly, so each
surviving monomial x^i y^j z^k r^(2s) (i + j + k + 2s = l) becomes
x^i y^j z^k / r^(2 nn + 1) with nn = l - s, and cc = coefficient /
((-1)^nn (2nn-1)!!).  Terms are ordered by l, then m = -l..l, then
lexicographically by (i, j, k); this reproduces the (i, j, k, nn) sequence of
the reference's unrolled l <= 6 kernel
(fast_rap_src_dfpt_gpu_eval/sum_up_far_dist_potential_dot.hpp:12-210) and its
logged counts n_cc_lm_ijk = 1, 4, 12, 28, 57, 104, 176 (280 at l = 7).

Polynomial algebra is exact (fractions); only the final normalisation uses
floating point.
"""

from __future__ import annotations

import math
from fractions import Fraction
from functools import lru_cache

import numpy as np

Poly = dict  # {(a, b, c): Fraction} for the monomial x^a y^b z^c


def _padd(p: Poly, q: Poly, scale=Fraction(1)) -> Poly:
    out = dict(p)
    for key, v in q.items():
        out[key] = out.get(key, Fraction(0)) + scale * v
        if out[key] == 0:
            del out[key]
    return out


def _pmul(p: Poly, q: Poly) -> Poly:
    out: Poly = {}
    for (a1, b1, c1), v1 in p.items():
        for (a2, b2, c2), v2 in q.items():
            key = (a1 + a2, b1 + b2, c1 + c2)
            out[key] = out.get(key, Fraction(0)) + v1 * v2
    return {k: v for k, v in out.items() if v != 0}


_X: Poly = {(1, 0, 0): Fraction(1)}
_Y: Poly = {(0, 1, 0): Fraction(1)}
_Z: Poly = {(0, 0, 1): Fraction(1)}
_R2: Poly = {(2, 0, 0): Fraction(1), (0, 2, 0): Fraction(1), (0, 0, 2): Fraction(1)}
_ONE: Poly = {(0, 0, 0): Fraction(1)}


@lru_cache(maxsize=None)
def _cs(m: int):
    """C_m + i S_m = (x + i y)^m as exact polynomials."""
    c, s = dict(_ONE), {}
    for _ in range(m):
        c, s = _padd(_pmul(_X, c), _pmul(_Y, s), Fraction(-1)), _padd(_pmul(_X, s), _pmul(_Y, c))
    return c, s


@lru_cache(maxsize=None)
def _q(l: int, m: int) -> Poly:
    """r^(l-m) Q_l^m(z/r): the Legendre recursion without Condon-Shortley phase,
    written homogeneously in (x, y, z)."""
    if l == m:
        return {(0, 0, 0): Fraction(math.prod(range(1, 2 * m, 2)) if m > 0 else 1)}
    if l == m + 1:
        return {k: v * (2 * m + 1) for k, v in _pmul(_Z, _q(m, m)).items()}
    a = {k: v * (2 * l - 1) for k, v in _pmul(_Z, _q(l - 1, m)).items()}
    b = {k: v * (l + m - 1) for k, v in _pmul(_R2, _q(l - 2, m)).items()}
    out = _padd(a, b, Fraction(-1))
    return {k: v / (l - m) for k, v in out.items()}


def solid_harmonic(l: int, m: int):
    """R_lm = r^l Y_lm as (normalisation float, exact polynomial)."""
    am = abs(m)
    ratio = Fraction(math.factorial(l - am), math.factorial(l + am))
    norm = math.sqrt((2 * l + 1) / (4.0 * math.pi) * float(ratio))
    c, s = _cs(am)
    if m == 0:
        poly = _q(l, 0)
    elif m > 0:
        norm *= math.sqrt(2.0)
        poly = _pmul(_q(l, am), c)
        if am & 1:
            poly = {k: -v for k, v in poly.items()}
    else:
        norm *= math.sqrt(2.0)
        poly = _pmul(_q(l, am), s)
    return norm, poly


def _eliminate_x2(poly: Poly):
    """Rewrite with x^2 -> r^2 - y^2 - z^2 until x is at most linear.
    Returns {(i, j, k, s): Fraction} for x^i y^j z^k r^(2s)."""
    work = {(a, b, c, 0): v for (a, b, c), v in poly.items()}
    done: dict = {}
    while work:
        (a, b, c, s), v = work.popitem()
        if a < 2:
            done[(a, b, c, s)] = done.get((a, b, c, s), Fraction(0)) + v
            continue
        for key, coef in (((a - 2, b, c, s + 1), v), ((a - 2, b + 2, c, s), -v), ((a - 2, b, c + 2, s), -v)):
            work[key] = work.get(key, Fraction(0)) + coef
            if work[key] == 0:
                del work[key]
    return {k: v for k, v in done.items() if v != 0}


def _double_factorial_odd(n: int) -> int:
    """(2n-1)!! with (-1)!! = 1."""
    return math.prod(range(1, 2 * n, 2)) if n > 0 else 1


@lru_cache(maxsize=None)
def multipole_tables(l_max_analytic_multipole: int):
    """Tables in the reference's layout for l <= l_max_analytic_multipole.

    Returns (index_cc, cc, n_cc_lm_ijk, index_ijk_max_cc) where index_cc is
    int32 (index_cc_dim_0, 6) Fortran-ordered (columns l, m, i, j, k, nn), cc is
    float64 (index_cc_dim_0,), n_cc_lm_ijk int32 (L+1,) cumulative term counts
    and index_ijk_max_cc int32 (3, L+1) the largest power of x, y, z used by
    any term with l' <= l.
    """
    L = l_max_analytic_multipole
    rows, coeffs, counts = [], [], []
    for l in range(L + 1):
        for m in range(-l, l + 1):
            norm, poly = solid_harmonic(l, m)
            terms = _eliminate_x2(poly)
            for (i, j, k, s) in sorted(terms, key=lambda t: (t[0], t[1], t[2])):
                nn = l - s
                assert 2 * nn == l + i + j + k
                rows.append((l, m, i, j, k, nn))
                coeffs.append(norm * float(terms[(i, j, k, s)]) / ((-1) ** nn * _double_factorial_odd(nn)))
        counts.append(len(rows))
    index_cc = np.asfortranarray(np.array(rows, dtype=np.int32))
    cc = np.array(coeffs, dtype=np.float64)
    n_cc = np.array(counts, dtype=np.int32)
    ijk_max = np.zeros((3, L + 1), dtype=np.int32, order="F")
    running = np.zeros(3, dtype=np.int32)
    start = 0
    for l in range(L + 1):
        for n in range(start, counts[l]):
            running = np.maximum(running, index_cc[n, 2:5])
        ijk_max[:, l] = running
        start = counts[l]
    return index_cc, cc, n_cc, ijk_max


def lm_index(l: int, m: int) -> int:
    """0-based position of (l, m) in a multipole_moments column (l*l + l + m),
    the reference's index_lm(m, l) - 1 (sum_up_whole_potential.cpp:349-356)."""
    return l * l + l + m
