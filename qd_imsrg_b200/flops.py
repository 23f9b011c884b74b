"""Algorithmic FP64 work of one IM-SRG(2) commutator, counted the way the
reference computes it (src/commutators.f90): every dgemm the reference calls
at 2*M*N*K flops, and the v_elem contractions of commutator_121/122 at
2 flops per non-vanishing term (terms whose two pairs sit in different
(M_L,M_S) blocks are exact zeros and are not counted).

These counts are the numerators of the TFLOP/s figures; the engine itself
does less work where it can (one Pandya product instead of two, known-zero
operator parts skipped), which is what a higher TFLOP/s then reflects.
"""
from __future__ import annotations

import numpy as np


def _gemm(M, N, K):
    return 2.0 * M * N * K


def states(emax: int) -> np.ndarray:
    """arrange_states (src/ME_general.f90:688-716): (n, ml, ms) per state."""
    out = []
    for R in range(emax):
        for ml in range(-R, R + 1, 2):
            for ms in (-1, 1):
                out.append(((R - abs(ml)) // 2, ml, ms))
    return np.array(out, dtype=np.int64)


def commutator_flops_parts(layout) -> dict:
    """Work split as the block sampler of the CPU baseline splits it:
    'onebody' (E0 and the one-body parts: 110, 220, 111, 121, 221),
    'block' (per (M_L,M_S) block: 122 and the matrix_mult222 ladders) and
    'cc' (per cross-coupled block, in build_cross_coupled order: the two
    construct_cc_ints products); plus the named components."""
    n, m = layout.nbody, layout.msp
    mp = m - n
    f = {}
    f["c110"] = _gemm(mp, mp, n)
    f["c111"] = (_gemm(n, n, n) + _gemm(n, n, mp) + _gemm(mp, mp, mp) + _gemm(mp, mp, n) +
                 2 * _gemm(mp, n, n) + 2 * _gemm(mp, n, mp))
    c220 = c221 = 0.0
    lad = np.zeros(layout.nblock)
    for q in range(layout.nblock):
        nh, nb, npp = (float(x) for x in layout.dims[q, :3])
        if npp * nh:
            c220 += _gemm(npp, npp, nh)
        # commutator_221 intermediates (commutators.f90:234-274)
        if npp * nh:
            c221 += _gemm(npp, npp, nh) + _gemm(nh, nh, npp)
        if npp * nb:
            c221 += _gemm(nb, nb, npp)
        if nh * nb:
            c221 += _gemm(nb, nb, nh)
        if nh * nb * npp:
            c221 += 2 * _gemm(nb, nh, npp) + 2 * _gemm(npp, nb, nh)
        # matrix_mult222 (commutators.f90:996-1130)
        x = 0.0
        if nh * npp:
            x += _gemm(nh, nh, npp) + _gemm(npp, npp, nh) + 2 * _gemm(npp, nh, npp) + 2 * _gemm(npp, nh, nh)
        if nh:
            x += _gemm(nh, nh, nh)
        if npp:
            x += _gemm(npp, npp, npp)
        if nb * npp * nh:
            x += 2 * _gemm(nb, nh, npp) + 2 * _gemm(npp, nb, nh)
        if nb * nh:
            x += 2 * _gemm(nb, nh, nh) + _gemm(nb, nb, nh)
        if nb * npp:
            x += 2 * _gemm(npp, nb, npp) + _gemm(nb, nb, npp)
        lad[q] = x
    f["c220"] = c220
    f["c221"] = c221
    f["ladder"] = float(lad.sum())
    # construct_cc_ints: two (r x r x nb) dgemms per cross-coupled block, in
    # the order of build_cross_coupled (ME_general.f90:380-381)
    qn = states(layout.emax)
    ml, ms = qn[:, 1], qn[:, 2]
    mlmax = 2 * int(ml.max())
    dml = ml[:, None] - ml[None, :]
    dms = ms[:, None] - ms[None, :]
    ccidx = (dml + mlmax) * 5 + (dms + 2)
    ncc = 10 * mlmax + 5
    r = np.bincount(ccidx.ravel(), minlength=ncc).astype(float)
    hp = np.zeros((m, m), bool)
    hp[:n, n:] = True
    nbcc = np.bincount(ccidx.ravel(), weights=hp.ravel().astype(float), minlength=ncc)
    cc = 2 * _gemm(r, r, nbcc)
    f["pandya"] = float(cc.sum())
    # commutator_121: per one-body target (x,y): (|HP(d)| + |HP(-d)|) terms, 2 operators
    neg = (-dml + mlmax) * 5 + (-dms + 2)
    f["c121"] = float(2 * 2 * (nbcc[ccidx] + nbcc[neg]).sum())
    # commutator_122: per stored element, 4 legs, |group(leg)| - 1 terms, 2 operators
    g = ml * 8 + ms
    gsize = {}
    for k in g:
        gsize[int(k)] = gsize.get(int(k), 0) + 1
    gs = np.array([gsize[int(k)] for k in g], dtype=float)
    c122 = np.zeros(layout.nblock)
    for q in range(layout.nblock):
        lists = [layout.pairs(q, k) - 1 for k in range(3)]
        legsum = [gs[p[:, 0]] + gs[p[:, 1]] - 2 if len(p) else np.zeros(0) for p in lists]
        t = 0.0
        for cb, ck in ((0, 0), (2, 2), (2, 0), (1, 1), (2, 1), (1, 0)):
            sb, sk = legsum[cb], legsum[ck]
            if len(sb) and len(sk):
                t += len(sk) * sb.sum() + len(sb) * sk.sum()
        c122[q] = 2 * 2 * t
    f["c122"] = float(c122.sum())
    f["total"] = float(sum(v for k, v in f.items()))
    onebody = f["c110"] + f["c220"] + f["c111"] + f["c121"] + f["c221"]
    return {"flops": f, "onebody": onebody, "block": c122 + lad, "cc": cc}


def commutator_flops(layout) -> dict:
    """{component: flops} and 'total' for [A,B] on a qd_imsrg_b200.Layout (or
    any object with nbody, msp, emax, nblock, dims[:, :3] = nhh, nph, npp and
    pairs(q, kind) giving 1-based pairs)."""
    return commutator_flops_parts(layout)["flops"]
