"""The closed forms of commutator_122 for a generator-like A (one-body part
fph only, two-body part Vpphh only: the Magnus generator Omega, the White
generator eta), which k_122_pppp and k_122_gen evaluate on the device, written
out in numpy and compared with the oracle's literal commutator_122
(commutators.f90:355-676) on every stored two-body part, for both herm
signs of B.  CPU only: this pins the formulas themselves; the GPU tests
compare the kernels with the oracle.

Notation: fA, fB are the fph parts of A and B, fppB, fhhB B's pp and hh
one-body parts, s the ordering sign of a pair, t runs over one (m_l, m_s)
group's holes or particles, pairs are indexed within their block."""
import numpy as np
import pytest

import oracle
from helpers import numpy_random_op


def _generator_like(O, vec):
    n, m = O.n, O.m
    mp = m - n
    out = np.zeros_like(vec)
    o = 1 + n * n + mp * mp
    out[o:o + mp * n] = vec[o:o + mp * n]
    for q in range(O.nblock):
        nh, npp = int(O.dims[q][0]), int(O.dims[q][2])
        s = int(O.offs[q][2])
        out[s:s + npp * nh] = vec[s:s + npp * nh]
    return out


def _closed_forms(O, a, hA, b, hB):
    """{(block, slot): matrix} of C = [A, B]_122 by the closed forms."""
    n, m = O.n, O.m
    mp = m - n
    o_fpp, o_fph = 1 + n * n, 1 + n * n + mp * mp
    fA = a[o_fph:o_fph + mp * n].reshape(n, mp).T  # fA[p - n, h] (0-based), states 1-based below
    fB = b[o_fph:o_fph + mp * n].reshape(n, mp).T
    fhhB = b[1:1 + n * n].reshape(n, n).T
    fppB = b[o_fpp:o_fpp + mp * mp].reshape(mp, mp).T
    qn = O.qn
    gid = {}
    grp = [gid.setdefault((qn[s][1], qn[s][2]), len(gid)) for s in range(m)]
    members = {}
    for s in range(m):
        members.setdefault(grp[s], []).append(s + 1)

    def holes(x):
        return [t for t in members[grp[x - 1]] if t <= n]

    def parts(x):
        return [t for t in members[grp[x - 1]] if t > n]

    def FA(pt, h):
        return fA[pt - n - 1, h - 1]

    def FB(pt, h):
        return fB[pt - n - 1, h - 1]

    out = {}
    for q in range(O.nblock):
        nh, nb, npp = (int(x) for x in O.dims[q, :3])
        hh, ph, pp = (O.pairs(q + 1, k) for k in range(3))
        ihh, iph, ipp = ({(int(x), int(y)): i for i, (x, y) in enumerate(L)} for L in (hh, ph, pp))

        def blk(v, slot, r, c):
            s0 = int(O.offs[q, slot])
            return v[s0:s0 + r * c].reshape(c, r).T

        def srt(idx, u, v):
            if u == v:
                return None, 0.0
            return (idx[(u, v)], 1.0) if u < v else (idx[(v, u)], -1.0)

        B = {k: blk(b, k, r, c) for k, (r, c) in enumerate([(nh, nh), (npp, npp), (npp, nh), (nb, nb), (npp, nb),
                                                               (nb, nh)])}
        Apphh = blk(a, 2, npp, nh)
        # C_pppp = hB W^T - hA W
        if npp:
            W = np.zeros((npp, npp))
            for j, (x, y) in enumerate(pp):
                for t in holes(x):
                    W[:, j] += FA(x, t) * B[4][:, iph[(t, y)]]
                for t in holes(y):
                    W[:, j] -= FA(y, t) * B[4][:, iph[(t, x)]]
            out[(q, 1)] = hB * W.T - hA * W
        # C_ppph
        if npp and nb:
            Cm = np.zeros((npp, nb))
            for i, (x, y) in enumerate(pp):
                for t in holes(x):
                    Cm[i, :] += FA(x, t) * B[3][iph[(t, y)], :]
                for t in holes(y):
                    Cm[i, :] -= FA(y, t) * B[3][iph[(t, x)], :]
            for j, (h, p) in enumerate(ph):
                for t in parts(h):
                    c_, s = srt(ipp, t, p)
                    if c_ is not None:
                        Cm[:, j] -= s * FA(t, h) * B[1][:, c_]
                for t in holes(p):
                    c_, s = srt(ihh, h, t)
                    if c_ is not None:
                        Cm[:, j] -= s * (hA * FA(p, t) * B[2][:, c_] - hB * FB(p, t) * Apphh[:, c_])
            out[(q, 4)] = Cm
        # C_pphh
        if npp and nh:
            Cm = np.zeros((npp, nh))
            for i, (x, y) in enumerate(pp):
                for side in (0, 1):
                    u, v = (x, y) if side == 0 else (y, x)
                    for t in holes(u):
                        Cm[i, :] += (1 - 2 * side) * FA(u, t) * B[5][iph[(t, v)], :]
                    for t in parts(u):
                        r_, s = srt(ipp, t, v) if side == 0 else srt(ipp, v, t)
                        if r_ is not None:
                            Cm[i, :] -= hB * s * fppB[t - n - 1, u - n - 1] * Apphh[r_, :]
            for j, (k1, k2) in enumerate(hh):
                for side in (0, 1):
                    kk, ko = (k1, k2) if side == 0 else (k2, k1)
                    for t in parts(kk):
                        Cm[:, j] += (1 - 2 * side) * FA(t, kk) * B[4][:, iph[(ko, t)]]
                    for t in holes(kk):
                        c_, s = srt(ihh, t, ko) if side == 0 else srt(ihh, ko, t)
                        if c_ is not None:
                            Cm[:, j] += hB * s * fhhB[kk - 1, t - 1] * Apphh[:, c_]
            out[(q, 2)] = Cm
        # C_phhh
        if nb and nh:
            Cm = np.zeros((nb, nh))
            for i, (h, p) in enumerate(ph):
                for t in parts(h):
                    r_, s = srt(ipp, t, p)
                    if r_ is not None:
                        Cm[i, :] += s * (hA * FA(t, h) * B[2][r_, :] - hB * FB(t, h) * Apphh[r_, :])
                for t in holes(p):
                    r_, s = srt(ihh, h, t)
                    if r_ is not None:
                        Cm[i, :] += s * FA(p, t) * B[0][r_, :]
            for j, (k1, k2) in enumerate(hh):
                for t in parts(k1):
                    Cm[:, j] += FA(t, k1) * B[3][:, iph[(k2, t)]]
                for t in parts(k2):
                    Cm[:, j] -= FA(t, k2) * B[3][:, iph[(k1, t)]]
            out[(q, 5)] = Cm
        # C_phph
        if nb:
            Cm = np.zeros((nb, nb))
            for i, (h, p) in enumerate(ph):
                for t in parts(h):
                    r_, s = srt(ipp, t, p)
                    if r_ is not None:
                        Cm[i, :] += hA * s * FA(t, h) * B[4][r_, :]
                for t in holes(p):
                    r_, s = srt(ihh, h, t)
                    if r_ is not None:
                        Cm[i, :] += hB * s * FA(p, t) * B[5][:, r_]
            for j, (k1, k2) in enumerate(ph):
                for t in parts(k1):
                    c_, s = srt(ipp, t, k2)
                    if c_ is not None:
                        Cm[:, j] -= hB * s * FA(t, k1) * B[4][c_, :]
                for t in holes(k2):
                    c_, s = srt(ihh, k1, t)
                    if c_ is not None:
                        Cm[:, j] -= hA * s * FA(k2, t) * B[5][:, c_]
            out[(q, 3)] = Cm
        # C_hhhh
        if nh and nb:
            Cm = np.zeros((nh, nh))
            for i, (b1, b2) in enumerate(hh):
                for t in parts(b1):
                    Cm[i, :] -= hA * FA(t, b1) * B[5][iph[(b2, t)], :]
                for t in parts(b2):
                    Cm[i, :] += hA * FA(t, b2) * B[5][iph[(b1, t)], :]
            for j, (k1, k2) in enumerate(hh):
                for t in parts(k1):
                    Cm[:, j] += hB * FA(t, k1) * B[5][iph[(k2, t)], :]
                for t in parts(k2):
                    Cm[:, j] -= hB * FA(t, k2) * B[5][iph[(k1, t)], :]
            out[(q, 0)] = Cm
        elif nh:
            out[(q, 0)] = np.zeros((nh, nh))
    return out


@pytest.mark.parametrize("n,R,hB", [(6, 5, 1), (6, 5, -1), (2, 5, 1), (12, 6, 1)])
def test_closed_forms_equal_commutator_122(n, R, hB):
    O = oracle.Layout(n, R)
    rng = np.random.default_rng(40 + n + R + hB)
    b = numpy_random_op(O, hB, rng, conserve=False)
    a = _generator_like(O, numpy_random_op(O, -1, rng))
    A, B, C = oracle.Op(O, -1, a), oracle.Op(O, hB, b), oracle.Op(O, 1)
    oracle.commutator_122(A, B, C)
    c = C.get()
    got = _closed_forms(O, a, -1.0, b, float(hB))
    seen = set()
    for (q, slot), M in got.items():
        r, cc = M.shape
        s0 = int(O.offs[q, slot])
        ref = c[s0:s0 + r * cc].reshape(cc, r).T
        assert np.abs(M - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max()), (q, slot)
        seen.add(slot)
    assert seen == {0, 1, 2, 3, 4, 5}
