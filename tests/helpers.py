"""Test helpers: comparison of vectorize-order operators part by part."""
import numpy as np

PART_NAMES = ["Vhhhh", "Vpppp", "Vpphh", "Vphph", "Vppph", "Vphhh"]


def part_slices(layout):
    """[(name, index array)] of the one-body and two-body parts of a layout
    (oracle.Layout or qd_imsrg_b200.Layout; both expose dims/offs/nbody)."""
    n = getattr(layout, "nbody", getattr(layout, "n", None))
    m = getattr(layout, "msp", getattr(layout, "m", None))
    mp = m - n
    out = [("E0", np.array([0]))]
    o = 1
    out.append(("fhh", np.arange(o, o + n * n))); o += n * n
    out.append(("fpp", np.arange(o, o + mp * mp))); o += mp * mp
    out.append(("fph", np.arange(o, o + mp * n))); o += mp * n
    idx = {k: [] for k in PART_NAMES}
    for q in range(layout.nblock):
        nh, nb, npp = (int(x) for x in layout.dims[q, :3])
        sizes = [nh * nh, npp * npp, npp * nh, nb * nb, npp * nb, nb * nh]
        for k, (name, sz) in enumerate(zip(PART_NAMES, sizes)):
            if sz:
                st = int(layout.offs[q, k])
                idx[name].append(np.arange(st, st + sz))
    for name in PART_NAMES:
        out.append((name, np.concatenate(idx[name]) if idx[name] else np.zeros(0, np.int64)))
    return out


def compare_parts(layout, got, ref, rtol=1e-12, atol_floor=1e-300, atol=None):
    """Relative Frobenius error per part; returns {name: (rel, maxabs)} and
    raises AssertionError listing parts above rtol.  With atol, a part whose
    max |diff| is at most atol also passes (for parts that are analytically
    zero and hold only rounding noise)."""
    res, bad = {}, []
    for name, ix in part_slices(layout):
        if ix.size == 0:
            continue
        d = got[ix] - ref[ix]
        nr = np.linalg.norm(ref[ix])
        rel = np.linalg.norm(d) / max(nr, atol_floor)
        mx = float(np.abs(d).max())
        res[name] = (rel, mx)
        if nr == 0.0:
            if mx > 1e-13:
                bad.append("%s: ref is zero, max|diff|=%.3e" % (name, mx))
        elif rel > rtol and not (atol is not None and mx <= atol):
            bad.append("%s: rel %.3e max %.3e" % (name, rel, mx))
    assert not bad, "; ".join(bad)
    return res


def numpy_random_op(L, herm, rng, conserve=True, sigma=0.1):
    """Independent numpy generator of a test operator for an oracle.Layout:
    N(0, sigma^2) entries, diagonal-class blocks (X + herm X^T)/2, E0 = 0."""
    v = rng.normal(0.0, sigma, L.neq)
    v[0] = 0.0
    n, m = L.n, L.m
    mp = m - n

    def sym(o, k):
        A = v[o:o + k * k].reshape(k, k, order="F")
        v[o:o + k * k] = ((A + herm * A.T) / 2).reshape(-1, order="F")

    sym(1, n)
    sym(1 + n * n, mp)
    if conserve:
        g = L.qn[:, 1] * 10 + L.qn[:, 2]
        o = 1
        F = v[o:o + n * n].reshape(n, n, order="F").copy(); F[g[:n, None] != g[None, :n]] = 0
        v[o:o + n * n] = F.reshape(-1, order="F"); o += n * n
        F = v[o:o + mp * mp].reshape(mp, mp, order="F").copy(); F[g[n:, None] != g[None, n:]] = 0
        v[o:o + mp * mp] = F.reshape(-1, order="F"); o += mp * mp
        F = v[o:o + mp * n].reshape(mp, n, order="F").copy(); F[g[n:, None] != g[None, :n]] = 0
        v[o:o + mp * n] = F.reshape(-1, order="F")
    for q in range(L.nblock):
        nh, nb, npp = (int(x) for x in L.dims[q, :3])
        oh, opp, _, oph = (int(x) for x in L.offs[q, :4])
        if nh:
            sym(oh, nh)
        if npp:
            sym(opp, npp)
        if nb:
            sym(oph, nb)
    return v


def synth_hamiltonian(L, rng, gap=2.0, vs=0.05, fs=0.05):
    """A Hermitian test Hamiltonian on which the Magnus flow converges:
    oscillator single-particle energies (holes lowered by `gap`) on the
    one-body diagonal, off-diagonal one-body entries ~ N(0, fs^2), two-body
    entries ~ N(0, vs^2), E0 = 0."""
    v = numpy_random_op(L, 1, rng, conserve=True, sigma=vs)
    n, m = L.n, L.m
    mp = m - n
    e = 2 * L.qn[:, 0] + np.abs(L.qn[:, 1]) + 1.0
    o = 1
    F = v[o:o + n * n].reshape(n, n, order="F") * (fs / vs)
    F[np.diag_indices(n)] = e[:n] - gap
    v[o:o + n * n] = F.reshape(-1, order="F")
    o += n * n
    F = v[o:o + mp * mp].reshape(mp, mp, order="F") * (fs / vs)
    F[np.diag_indices(mp)] = e[n:]
    v[o:o + mp * mp] = F.reshape(-1, order="F")
    o += mp * mp
    v[o:o + mp * n] *= fs / vs
    v[0] = 0.0
    return v



def eom_scalar_positions(O):
    """Positions in the vectorize array of the scalar-target EOM vector's
    entries, in the reference's unwrap order (EOM_IMSRG.f90:815-884): the
    1p1h entries in fph, then the 2p2h entries in each block's Vpphh.
    O: an oracle.Layout (the library's layout has the same blocks)."""
    n, m = O.n, O.m
    mp = m - n
    qn = O.qn
    pp, hh = {}, {}
    for q in range(O.nblock):
        for k, (a, b) in enumerate(O.pairs(q + 1, 2)):
            pp[(int(a), int(b))] = (q, k)
        for k, (i, j) in enumerate(O.pairs(q + 1, 0)):
            hh[(int(i), int(j))] = (q, k)
    o_fph = 1 + n * n + mp * mp
    pos = [o_fph + (a - n - 1) + (i - 1) * mp for a in range(n + 1, m + 1) for i in range(1, n + 1)
           if tuple(qn[a - 1][1:]) == tuple(qn[i - 1][1:])]
    for a in range(n + 1, m + 1):
        for b in range(a + 1, m + 1):
            qa = pp[(a, b)]
            for i in range(1, n + 1):
                for j in range(i + 1, n + 1):
                    qh = hh[(i, j)]
                    if qa[0] == qh[0]:
                        pos.append(int(O.offs[qa[0], 2]) + qa[1] + qh[1] * int(O.dims[qa[0], 2]))
    return np.array(pos, np.int64)
