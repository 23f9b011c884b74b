"""HQ_comm_1b / HQ_comm_2b (src/commutators.f90:1162-1272), the EOM-IMSRG
matrix-vector product, restated literally for small bases, as the checker of
qd_eom_matvec and qd_eom_matvec_target.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module.

States are 1-based as in the reference; operators are held in vectorize
order.  f_elem follows ME_general.f90:1780-1813, Qf_elem :1835-1870 (only
particle-hole entries), Q_elem :1170-1224 (only pphh entries, antisymmetric).
HQ reads Q from a blocked operator through v_elem, which carries the same
ordering signs (scalar target Mltarg = Mstarg = 0); HQTarget reads it from
the reference's own dense storage of a ladder operator of any target, and
matvec_prod restates EOM_IMSRG.f90:551-649 with unwrap / rewrap around it."""
from __future__ import annotations

import numpy as np

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


# ---------------------------------------------------------------------------
# Any target (Mltarg, Mstarg): the ladder operator is stored as the reference
# stores it (allocate_ex): fph(m-n, n) and one matrix mat(1)%Vpphh over all
# particle pairs x all hole pairs, indexed by fermionic_tp_index.

def tp_index(i, j, n):  # fermionic_tp_index, ME_general.f90:1348-1357 (i < j, 1-based)
    return n * (i - 1) + (i - i * i) // 2 + j - i


class HQTarget(HQ):
    """HQ_comm_1b / HQ_comm_2b with Qf_elem (ME_general.f90:1835-1870) and
    Q_elem (ME_general.f90:1170-1224) reading the reference's dense storage."""

    def __init__(self, O, Hop, hvec, hherm, fph, vpp):
        super().__init__(O, Hop, hvec, hherm, None, None)
        self.fph, self.vpp = fph, vpp

    def qf(self, a, b):
        if a > self.n and b <= self.n:
            return self.fph[a - self.n - 1, b - 1]
        return 0.0

    def q(self, a, b, c, d):
        N = self.n
        if a == b or c == d or a <= N or b <= N or c > N or d > N:
            return 0.0
        pre = 1.0
        if a > b:
            a, b, pre = b, a, -pre
        if c > d:
            c, d, pre = d, c, -pre
        return self.vpp[tp_index(a - N, b - N, self.mp) - 1, tp_index(c, d, N) - 1] * pre


def _targets(O, ml, ms):
    """The 1p1h (ix, jx) and 2p2h (a, b, i, j) index tuples of the target in
    unwrap order (EOM_IMSRG.f90:815-884), 1-based particle / hole indices."""
    n, p = O.n, O.m - O.n
    qn = O.qn
    L = lambda s: qn[s - 1][1]
    S = lambda s: qn[s - 1][2]
    one = [(ix, jx) for ix in range(1, p + 1) for jx in range(1, n + 1)
           if L(n + ix) - L(jx) == ml and S(n + ix) - S(jx) == ms]
    two = [(a, b, i, j) for a in range(1, p + 1) for b in range(a + 1, p + 1)
           for i in range(1, n + 1) for j in range(i + 1, n + 1)
           if L(n + a) + L(n + b) - L(i) - L(j) == ml and S(n + a) + S(n + b) - S(i) - S(j) == ms]
    return one, two


def eom_dim(O, ml, ms):
    one, two = _targets(O, ml, ms)
    return len(one), len(two)


def unwrap(O, ml, ms, v):
    """EOM_IMSRG.f90:815-884: v -> (fph, Vpphh) of the ladder operator."""
    n, p = O.n, O.m - O.n
    one, two = _targets(O, ml, ms)
    fph = np.zeros((p, n))
    vpp = np.zeros((p * (p - 1) // 2, n * (n - 1) // 2))
    g = 0
    for ix, jx in one:
        fph[ix - 1, jx - 1] = v[g]
        g += 1
    for a, b, i, j in two:
        vpp[tp_index(a, b, p) - 1, tp_index(i, j, n) - 1] = v[g]
        g += 1
    return fph, vpp


def matvec_prod(O, Hop, hvec, hherm, ml, ms, v):
    """matvec_prod (EOM_IMSRG.f90:551-649): unwrap v, HQ_comm_1b on the
    target's 1p1h entries, HQ_comm_2b on its 2p2h entries, rewrap
    (EOM_IMSRG.f90:1011-1080, the same order as unwrap)."""
    n = O.n
    fph, vpp = unwrap(O, ml, ms, v)
    r = HQTarget(O, Hop, hvec, hherm, fph, vpp)
    one, two = _targets(O, ml, ms)
    w = np.empty(len(one) + len(two))
    g = 0
    for ix, jx in one:
        w[g] = r.comm_1b(ix + n, jx)
        g += 1
    for a, b, i, j in two:
        w[g] = r.comm_2b(a + n, b + n, i, j)
        g += 1
    return w
