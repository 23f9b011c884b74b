"""HQ_comm_1b / HQ_comm_2b (src/commutators.f90:1162-1272), the EOM-IMSRG
matrix-vector product, restated literally for small bases, as the checker of
qd_eom_matvec.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module.

States are 1-based as in the reference; operators are held in vectorize
order.  f_elem follows ME_general.f90:1780-1813, Qf_elem :1835-1870 (only
particle-hole entries), Q_elem :1170-1224 (only pphh entries, antisymmetric;
read here from the blocked Vpphh through v_elem, which carries the same
ordering signs).  Only (M_L, M_S)-conserving excitations are compared (the
reference's scalar target Mltarg = Mstarg = 0)."""
from __future__ import annotations

from . import v_elem


class HQ:
    def __init__(self, O, Hop, hvec, hherm, Qop, qvec):
        self.O, self.H, self.Q = O, Hop, Qop
        self.hv, self.hh, self.qv = hvec, float(hherm), qvec
        n, m = O.n, O.m
        self.n, self.m, self.mp = n, m, m - n
        self.o_fhh, self.o_fpp = 1, 1 + n * n
        self.o_fph = self.o_fpp + self.mp * self.mp

    def f(self, a, b):
        n, mp = self.n, self.mp
        if a <= n:
            if b <= n:
                return self.hv[self.o_fhh + (a - 1) + (b - 1) * n]
            return self.hv[self.o_fph + (b - n - 1) + (a - 1) * mp] * self.hh
        if b <= n:
            return self.hv[self.o_fph + (a - n - 1) + (b - 1) * mp]
        return self.hv[self.o_fpp + (a - n - 1) + (b - n - 1) * mp]

    def qf(self, a, b):
        if a > self.n and b <= self.n:
            return self.qv[self.o_fph + (a - self.n - 1) + (b - 1) * self.mp]
        return 0.0

    def q(self, a, b, c, d):
        n = self.n
        if a == b or c == d or a <= n or b <= n or c > n or d > n:
            return 0.0
        return v_elem(a, b, c, d, self.Q)

    def v(self, a, b, c, d):
        return v_elem(a, b, c, d, self.H)

    def comm_1b(self, a, i):  # commutators.f90:1162-1211
        N, M = self.n, self.m
        f, qf, q, v = self.f, self.qf, self.q, self.v
        sm = 0.0
        for b in range(N + 1, M + 1):
            sm += f(a, b) * qf(b, i)
        for j in range(1, N + 1):
            sm -= qf(a, j) * f(j, i)
        for b in range(N + 1, M + 1):
            for j in range(1, N + 1):
                sm += f(j, b) * q(a, b, i, j)
                sm += qf(b, j) * v(a, j, i, b)
        for b in range(N + 1, M + 1):
            for c in range(b + 1, M + 1):
                for j in range(1, N + 1):
                    sm += q(c, b, i, j) * v(a, j, c, b)
        for b in range(N + 1, M + 1):
            for k in range(1, N + 1):
                for j in range(k + 1, N + 1):
                    sm -= q(a, b, k, j) * v(k, j, i, b)
        return sm

    def comm_2b(self, a, b, i, j):  # commutators.f90:1214-1272
        N, M = self.n, self.m
        f, qf, q, v = self.f, self.qf, self.q, self.v
        sm = 0.0
        for c in range(N + 1, M + 1):
            sm += f(a, c) * q(c, b, i, j) - f(b, c) * q(c, a, i, j)
            sm += qf(c, i) * v(a, b, c, j) - qf(c, j) * v(a, b, c, i)
        for k in range(1, N + 1):
            sm += -q(a, b, k, j) * f(k, i) + q(a, b, k, i) * f(k, j)
            sm += -v(b, k, j, i) * qf(a, k) + v(a, k, j, i) * qf(b, k)
        for c in range(N + 1, M + 1):
            for d in range(c + 1, M + 1):
                sm += v(a, b, c, d) * q(c, d, i, j)
        for k in range(1, N + 1):
            for l in range(k + 1, N + 1):
                sm += v(k, l, i, j) * q(a, b, k, l)
        for k in range(1, N + 1):
            for c in range(N + 1, M + 1):
                sm -= v(b, k, c, i) * q(a, c, k, j)
                sm += v(a, k, c, i) * q(b, c, k, j)
                sm += v(b, k, c, j) * q(a, c, k, i)
                sm -= v(a, k, c, j) * q(b, c, k, i)
        return sm
