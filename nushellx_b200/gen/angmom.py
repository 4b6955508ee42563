"""Angular-momentum coupling coefficients (all arguments are TWICE the physical value).

Own implementation of the standard closed forms (Racah's formulas as given in
Edmonds, "Angular Momentum in Quantum Mechanics", eqs. 3.6.11 and 6.3.7), in
double precision with exact integer factorials.  The reference's equivalents are
``clebg`` (src/NuCommon/IClebg.FI) and ``sixj``/``racah``
(src/NuCommon/NuCommon.f90:3255-3309); the conventions below match them:

* ``cg(j1, j2, J, m1, m2, M)`` = <j1 m1 j2 m2 | J M> (Condon-Shortley phases);
* ``sixj(a, b, c, d, e, f)`` = {a b c; d e f};
* ``racah_w(j1, j2, j3, j4, J, K)`` = W(j1 j2 j3 j4; J K)
  = (-1)^((j1+j2+j3+j4)/2) {j1 j2 J; j4 j3 K}, as in NuCommon.f90:3255-3265.
"""
from functools import lru_cache
from math import factorial, sqrt


def _f(n2):
    """factorial of n2/2 (n2 even, >= 0)."""
    return factorial(n2 // 2)


def triangle(a, b, c):
    """True if (a/2, b/2, c/2) satisfy the triangle rule and parity (twice-values)."""
    return abs(a - b) <= c <= a + b and (a + b + c) % 2 == 0


@lru_cache(maxsize=None)
def cg(j1, j2, J, m1, m2, M):
    if m1 + m2 != M:
        return 0.0
    if not triangle(j1, j2, J):
        return 0.0
    if abs(m1) > j1 or abs(m2) > j2 or abs(M) > J:
        return 0.0
    if (j1 + m1) % 2 or (j2 + m2) % 2 or (J + M) % 2:
        return 0.0
    # Racah's closed form (Edmonds 3.6.11)
    pre = (J + 1) * _f(j1 + j2 - J) * _f(j1 - j2 + J) * _f(-j1 + j2 + J) / _f(j1 + j2 + J + 2)
    pre *= _f(j1 + m1) * _f(j1 - m1) * _f(j2 + m2) * _f(j2 - m2) * _f(J + M) * _f(J - M)
    s = 0.0
    kmin = max(0, j2 - J - m1, j1 + m2 - J)
    kmax = min(j1 + j2 - J, j1 - m1, j2 + m2)
    for k2 in range(kmin, kmax + 1, 2):
        den = (_f(k2) * _f(j1 + j2 - J - k2) * _f(j1 - m1 - k2) * _f(j2 + m2 - k2)
               * _f(J - j2 + m1 + k2) * _f(J - j1 - m2 + k2))
        s += (-1) ** (k2 // 2) / den
    return sqrt(pre) * s


def _delta(a, b, c):
    return _f(a + b - c) * _f(a - b + c) * _f(-a + b + c) / _f(a + b + c + 2)


@lru_cache(maxsize=None)
def sixj(a, b, c, d, e, f):
    """Wigner 6-j symbol {a b c; d e f} (Racah formula, Edmonds 6.3.7)."""
    for (x, y, z) in ((a, b, c), (a, e, f), (d, b, f), (d, e, c)):
        if not triangle(x, y, z):
            return 0.0
    pre = sqrt(_delta(a, b, c) * _delta(a, e, f) * _delta(d, b, f) * _delta(d, e, c))
    t_lo = max(a + b + c, a + e + f, d + b + f, d + e + c)
    t_hi = min(a + b + d + e, b + c + e + f, a + c + d + f)
    s = 0.0
    for t in range(t_lo, t_hi + 1, 2):
        num = (-1) ** (t // 2) * _f(t + 2)
        den = (_f(t - a - b - c) * _f(t - a - e - f) * _f(t - d - b - f) * _f(t - d - e - c)
               * _f(a + b + d + e - t) * _f(b + c + e + f - t) * _f(a + c + d + f - t))
        s += num / den
    return pre * s


def racah_w(j1, j2, j3, j4, J, K):
    """Racah W(j1 j2 j3 j4; J K) in the NuCommon.f90:3255 form."""
    ph = -1.0 if ((j1 + j2 + j3 + j4) // 2) % 2 else 1.0
    return ph * sixj(j1, j2, J, j4, j3, K)
