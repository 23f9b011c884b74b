"""Dense textbook IM-SRG(2) commutator, written independently of the reference.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module.

The blocked oracle (oracle.cpp) restates the reference's own loops, so it
inherits any slip the reference may contain.  This module is written from
the physics instead: the normal-ordered commutator [A, B] of two operators
with zero-, one- and two-body parts, truncated at two-body, on full m x m and
m^4 antisymmetric tensors.  The formulas are the fundamental commutators of
the IM-SRG(2) (Hergert, Bogner, Morris, Schwenk, Tsukiyama, Phys. Rep. 621
(2016) 165, the flow equations written for a general pair A, B):

  C0      = sum_ab (n_a - n_b) A_ab B_ba
            + 1/4 sum_abcd (A_abcd B_cdab - B_abcd A_cdab) n_a n_b nb_c nb_d
  C_12    = sum_a (A_1a B_a2 - B_1a A_a2)
            + sum_ab (n_a - n_b) (A_ab B_b1a2 - B_ab A_b1a2)
            + 1/2 sum_abc (n_a n_b nb_c + nb_a nb_b n_c) (A_c1ab B_abc2 - B_c1ab A_abc2)
  C_1234  = sum_a (1 - P_12) (A_1a B_a234 - B_1a A_a234)
            - sum_a (1 - P_34) (A_a3 B_12a4 - B_a3 A_12a4)
            + 1/2 sum_ab (1 - n_a - n_b) (A_12ab B_ab34 - B_12ab A_ab34)
            - sum_ab (n_a - n_b) (1 - P_12)(1 - P_34) A_b2a4 B_a1b3

with n_p the reference occupation (1 for the N lowest states, the holes) and
nb_p = 1 - n_p.  The last line is the particle-hole (Pandya) channel; the
reference's Magnus driver omits it, so `commutator` takes `pandya`.

Conversion to and from the reference's vectorize order uses only the
storage rules of the blocked layout (ME_general.f90:1871-1989 vectorize,
:1557-1680 v_elem, :1780-1813 f_elem): stored classes hh-hh, pp-pp, pp-hh,
ph-ph, pp-ph, ph-hh per (M_L, M_S) block, ph pairs as (hole, particle), the
transposed classes as herm times the transpose, and zero across blocks.
"""
from __future__ import annotations

import numpy as np

# (row pair kind, column pair kind) of the six stored sub-blocks, in the
# column order of the layout's offsets; kind 0 = hh, 1 = ph, 2 = pp
_CLASSES = [(0, 0), (2, 2), (2, 0), (1, 1), (2, 1), (1, 0)]


def _one_body_slices(n: int, m: int):
    mp = m - n
    o = 1
    s_hh = slice(o, o + n * n); o += n * n
    s_pp = slice(o, o + mp * mp); o += mp * mp
    s_ph = slice(o, o + mp * n)
    return s_hh, s_pp, s_ph


def _pairs(L):
    """0-based pair arrays [q][kind] of an oracle.Layout."""
    return [[L.pairs(q, k).astype(np.int64) - 1 for k in range(3)] for q in range(1, L.nblock + 1)]


def to_dense(L, vec: np.ndarray, herm: int):
    """(E0, f[m,m], V[m,m,m,m]) of an operator stored in vectorize order."""
    n, m = L.n, L.m
    mp = m - n
    s_hh, s_pp, s_ph = _one_body_slices(n, m)
    f = np.zeros((m, m))
    f[:n, :n] = vec[s_hh].reshape(n, n, order="F")
    f[n:, n:] = vec[s_pp].reshape(mp, mp, order="F")
    fph = vec[s_ph].reshape(mp, n, order="F")
    f[n:, :n] = fph
    f[:n, n:] = herm * fph.T
    V = np.zeros((m, m, m, m))
    for q, P in enumerate(_pairs(L)):
        for k, (rk, ck) in enumerate(_CLASSES):
            R, Cc = P[rk], P[ck]
            if len(R) == 0 or len(Cc) == 0:
                continue
            o = int(L.offs[q, k])
            M = vec[o:o + len(R) * len(Cc)].reshape(len(R), len(Cc), order="F")
            _put(V, R, Cc, M)
            if rk != ck:
                _put(V, Cc, R, herm * M.T)
    return float(vec[0]), f, V


def _put(V, R, Cc, M):
    p, q = R[:, 0][:, None], R[:, 1][:, None]
    r, s = Cc[:, 0][None, :], Cc[:, 1][None, :]
    V[p, q, r, s] = M
    V[q, p, r, s] = -M
    V[p, q, s, r] = -M
    V[q, p, s, r] = M


def from_dense(L, E0: float, f: np.ndarray, V: np.ndarray) -> np.ndarray:
    """The stored entries of (E0, f, V) in vectorize order."""
    n, m = L.n, L.m
    vec = np.zeros(L.neq)
    vec[0] = E0
    s_hh, s_pp, s_ph = _one_body_slices(n, m)
    vec[s_hh] = f[:n, :n].reshape(-1, order="F")
    vec[s_pp] = f[n:, n:].reshape(-1, order="F")
    vec[s_ph] = f[n:, :n].reshape(-1, order="F")
    for q, P in enumerate(_pairs(L)):
        for k, (rk, ck) in enumerate(_CLASSES):
            R, Cc = P[rk], P[ck]
            if len(R) == 0 or len(Cc) == 0:
                continue
            o = int(L.offs[q, k])
            M = V[R[:, 0][:, None], R[:, 1][:, None], Cc[:, 0][None, :], Cc[:, 1][None, :]]
            vec[o:o + M.size] = M.reshape(-1, order="F")
    return vec


def _anti12(T):
    return T - T.transpose(1, 0, 2, 3)


def _anti34(T):
    return T - T.transpose(0, 1, 3, 2)


def commutator(A, B, occ: np.ndarray, pandya: bool = True):
    """Dense IM-SRG(2) [A, B]; A and B are (E0, f, V) triples."""
    _, fA, VA = A
    _, fB, VB = B
    m = fA.shape[0]
    n = occ.astype(np.float64)
    nb = 1.0 - n
    w = n[:, None] - n[None, :]  # n_a - n_b
    ee = np.einsum

    # zero-body
    c0 = float(np.sum(w * fA * fB.T))
    hhpp = n[:, None, None, None] * n[None, :, None, None] * nb[None, None, :, None] * nb[None, None, None, :]
    c0 += 0.25 * float(np.sum(hhpp * (VA * VB.transpose(2, 3, 0, 1) - VB * VA.transpose(2, 3, 0, 1))))

    # one-body
    c1 = fA @ fB - fB @ fA
    c1 += ee("ab,biaj->ij", w * fA, VB) - ee("ab,biaj->ij", w * fB, VA)
    W3 = (n[:, None, None] * n[None, :, None] * nb[None, None, :]
          + nb[:, None, None] * nb[None, :, None] * n[None, None, :])
    c1 += 0.5 * (ee("ciab,abc,abcj->ij", VA, W3, VB, optimize=True)
                 - ee("ciab,abc,abcj->ij", VB, W3, VA, optimize=True))

    # two-body
    c2 = _anti12(ee("ia,ajkl->ijkl", fA, VB) - ee("ia,ajkl->ijkl", fB, VA))
    c2 -= _anti34(ee("ak,ijal->ijkl", fA, VB) - ee("ak,ijal->ijkl", fB, VA))
    wl = (1.0 - n[:, None] - n[None, :]).reshape(-1)
    Am, Bm = VA.reshape(m * m, m * m), VB.reshape(m * m, m * m)
    c2 += 0.5 * ((Am * wl[None, :]) @ Bm - (Bm * wl[None, :]) @ Am).reshape(m, m, m, m)
    if pandya:
        G = ee("ab,bjal,aibk->ijkl", w, VA, VB, optimize=True)
        c2 -= _anti34(_anti12(G))
    return c0, c1, c2


def mbpt2(f: np.ndarray, V: np.ndarray, nbody: int) -> float:
    """Second-order energy 1/4 sum_abij |V_abij|^2 / (f_ii + f_jj - f_aa - f_bb)
    over holes i, j and particles a, b, with the diagonal of f as energies."""
    e = np.diag(f)
    eh, ep = e[:nbody], e[nbody:]
    den = eh[None, None, :, None] + eh[None, None, None, :] - ep[:, None, None, None] - ep[None, :, None, None]
    v = V[nbody:, nbody:, :nbody, :nbody]
    return 0.25 * float(np.sum(v * v / den))
