"""Exact error metrics (test infrastructure, never the product): the reference's
ground-truth metrics of src/runtime.cpp:194-242, evaluated in exact rational
arithmetic (every float64 is a binary rational, so the residual sums are exact)
with the final square roots and quotient in 60-digit decimal. Slow and meant for
small matrices; it pins the GPU double-double metrics independently of the
reference's long double, whose 64-bit sums lose digits on residuals near the
unit roundoff.

Only ``tests/`` import this module.
"""
import decimal
from fractions import Fraction

import numpy as np

_CTX = decimal.Context(prec=60)


def _sqrt(fr):
    return _CTX.sqrt(_CTX.divide(decimal.Decimal(fr.numerator), decimal.Decimal(fr.denominator)))


def _F(a):
    return [[Fraction(float(v)) for v in row] for row in a]


def solve_backward_error(A, x, b):
    out = []
    for a, xv, bv in zip(np.asarray(A, np.float64), np.asarray(x, np.float64), np.asarray(b, np.float64)):
        n = a.shape[0]
        af, xf, bf = _F(a), [Fraction(float(v)) for v in xv], [Fraction(float(v)) for v in bv]
        num = sum((bf[i] - sum(af[i][j] * xf[j] for j in range(n))) ** 2 for i in range(n))
        fa = sum(v * v for row in af for v in row)
        fx = sum(v * v for v in xf)
        fb = sum(v * v for v in bf)
        den = _CTX.add(_CTX.multiply(_sqrt(fa), _sqrt(fx)), _sqrt(fb))
        out.append(float(_CTX.divide(_sqrt(num), den)))
    return np.array(out)


def lu_backward_error(A, LU, piv):
    out = []
    for a, f, pv in zip(np.asarray(A, np.float64), np.asarray(LU, np.float64), np.asarray(piv)):
        n = a.shape[0]
        af, ff = _F(a), _F(f)
        perm = list(range(n))
        for k in range(n):
            perm[k], perm[pv[k]] = perm[pv[k]], perm[k]
        num = Fraction(0)
        for i in range(n):
            for j in range(n):
                s = sum(((Fraction(1) if k == i else ff[i][k]) * ff[k][j]) for k in range(min(i, j) + 1))
                num += (af[perm[i]][j] - s) ** 2
        fa = sum(v * v for row in af for v in row)
        out.append(float(_CTX.divide(_sqrt(num), _sqrt(fa))))
    return np.array(out)


def chol_backward_error(A, L):
    out = []
    for a, l in zip(np.asarray(A, np.float64), np.asarray(L, np.float64)):
        n = a.shape[0]
        af, lf = _F(a), _F(l)
        num = Fraction(0)
        for i in range(n):
            for j in range(n):
                s = sum(lf[i][k] * lf[j][k] for k in range(min(i, j) + 1))
                num += (af[i][j] - s) ** 2
        fa = sum(v * v for row in af for v in row)
        out.append(float(_CTX.divide(_sqrt(num), _sqrt(fa))))
    return np.array(out)
