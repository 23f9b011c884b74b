"""Exact rational evaluation of the 2-D oscillator Coulomb element v_int.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module.

The closed form is the one src/ME_general.f90:2205-2276 evaluates
(E. Anisimovas and A. Matulis, J. Phys.: Condens. Matter 10 (1998) 601):
two nested alternating sums of binomials, factorials and Gamma functions of
half-integers.  Here every sum is a Python Fraction, so nothing cancels
inexactly.  Two facts make the result rational up to one common factor:

* in the inner sum l4 = l1 + l2 - l3, so LAM = l1 + l2 + l3 + l4 is even and
  Gamma(1 + LAM/2) = (LAM/2)!;
* G = sum(gs) = 2 (j1 + j2 + j3 + j4) + |ml_i| + |ml_j| + |ml_k| + |ml_l|
  has one parity per element: for G odd every Gamma((G-LAM+1)/2) is a
  factorial and 0.5**((G+1)/2) is rational; for G even each term carries
  sqrt(pi) * 2**(-G/2) / sqrt(2), i.e. a common sqrt(pi/2).

The square roots (of pi/2, of the normalisation product and of hbar-omega)
are taken at the end in 60-digit decimal arithmetic.
"""
from __future__ import annotations

import math
from decimal import Decimal, localcontext
from fractions import Fraction
from functools import lru_cache

_PI = Decimal("3.14159265358979323846264338327950288419716939937510582097494459")


@lru_cache(maxsize=None)
def _sm_int(g0: int, g1: int, g2: int, g3: int) -> Fraction:
    G = g0 + g1 + g2 + g3
    tot = Fraction(0)
    for l1 in range(g0 + 1):
        for l2 in range(g1 + 1):
            for l3 in range(g2 + 1):
                l4 = l1 + l2 - l3
                if l4 < 0 or l4 > g3:
                    continue
                lam = l1 + l2 + l3 + l4
                sgn = -1 if (g1 + g2 - l2 - l3) & 1 else 1
                t = sgn * math.comb(g0, l1) * math.comb(g1, l2) * math.comb(g2, l3) * math.comb(g3, l4)
                t *= math.factorial(lam // 2)
                if G % 2 == 0:  # Gamma(k + 1/2) / sqrt(pi) = (2k)! / (4^k k!)
                    k = (G - lam) // 2
                    tot += Fraction(t * math.factorial(2 * k), 4 ** k * math.factorial(k))
                else:
                    tot += t * math.factorial((G - lam - 1) // 2)
    return tot


def v_int_exact(qi, qj, qk, ql, hw: float = 1.0) -> float:
    """v_int(qi, qj, qk, ql, hw) with q = (n, ml, ms), correctly rounded to
    double up to the final 60-digit square roots."""
    if not (qi[2] == ql[2] and qk[2] == qj[2]):
        return 0.0

    def up(m):
        return (abs(m) + m) // 2

    def dn(m):
        return (abs(m) - m) // 2

    sm = Fraction(0)
    even = (abs(qi[1]) + abs(qj[1]) + abs(qk[1]) + abs(ql[1])) % 2 == 0
    for j1 in range(qi[0] + 1):
        for j2 in range(qj[0] + 1):
            for j3 in range(qk[0] + 1):
                for j4 in range(ql[0] + 1):
                    g0 = j1 + j4 + up(qi[1]) + dn(ql[1])
                    g3 = j1 + j4 + dn(qi[1]) + up(ql[1])
                    g1 = j2 + j3 + up(qj[1]) + dn(qk[1])
                    g2 = j2 + j3 + dn(qj[1]) + up(qk[1])
                    G = g0 + g1 + g2 + g3
                    s4 = -1 if (j1 + j2 + j3 + j4) & 1 else 1
                    t = Fraction(s4, math.factorial(j1) * math.factorial(j2) * math.factorial(j3)
                                 * math.factorial(j4))
                    t *= math.comb(qi[0] + abs(qi[1]), qi[0] - j1) * math.comb(qj[0] + abs(qj[1]), qj[0] - j2)
                    t *= math.comb(qk[0] + abs(qk[1]), qk[0] - j3) * math.comb(ql[0] + abs(ql[1]), ql[0] - j4)
                    # 0.5**((G+1)/2): rational for G odd; 2**(-G/2) / sqrt(2) for G even
                    t *= Fraction(1, 2 ** ((G + 1) // 2)) if G % 2 else Fraction(1, 2 ** (G // 2))
                    sm += t * _sm_int(g0, g1, g2, g3)
    f = Fraction(1)
    for q in (qi, qj, qk, ql):
        f *= Fraction(math.factorial(q[0]), math.factorial(q[0] + abs(q[1])))
    with localcontext() as ctx:
        ctx.prec = 60
        val = Decimal(sm.numerator) / Decimal(sm.denominator)
        if even:
            val *= (_PI / 2).sqrt()
        val *= (Decimal(f.numerator) / Decimal(f.denominator)).sqrt() * Decimal(hw).sqrt()
        return float(val)
