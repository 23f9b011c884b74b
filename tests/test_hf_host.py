"""CPU checks of the host-side flow inputs: Coulomb TBMEs (v_int of the
reference, real(16) arithmetic kept, and its __float128 variant against an
exact rational evaluation) and Hartree-Fock, against closed-form and
published values for the 2-D quantum dot and against invariants."""
import math
import os

import numpy as np
import pytest

import qd_imsrg_b200 as qd


def test_v_int_lowest_orbital_closed_form():
    # <00,00|1/r|00,00> = sqrt(pi/2) in oscillator units (hbar-omega = 1)
    v = qd.v_int((0, 0, -1), (0, 0, -1), (0, 0, -1), (0, 0, -1), 1.0)
    assert v == pytest.approx(math.sqrt(math.pi / 2), rel=1e-15)
    # hbar-omega scaling sqrt(hw) (ME_general.f90:2267) and the spin selection
    assert qd.v_int((0, 0, -1), (0, 0, -1), (0, 0, -1), (0, 0, -1), 0.25) == pytest.approx(0.5 * v, rel=1e-15)
    assert qd.v_int((0, 0, -1), (0, 0, 1), (0, 0, -1), (0, 0, -1), 1.0) == 0.0


def test_v_int_symmetries():
    a, b, c, d = (0, 1, -1), (0, -1, -1), (1, 0, -1), (0, 0, -1)  # ml_a+ml_b = 0 = ml_c+ml_d
    # <ab|V|cd> = v_int(a,b,d,c); particle exchange and hermiticity
    v1 = qd.v_int(a, b, d, c)
    v2 = qd.v_int(b, a, c, d)   # <ba|dc>
    v3 = qd.v_int(c, d, b, a)   # <cd|ab>
    assert v1 == pytest.approx(v2, rel=1e-13) and v1 == pytest.approx(v3, rel=1e-13)
    assert abs(v1) > 1e-3


# (n, ml, ms) quadruples: low radial quantum numbers, where the reference's
# real(8) sums still hold ~12 digits, and high ones, where they hold none
LOW_N = [((0, 1, 1), (0, -1, -1), (0, -1, -1), (0, 1, 1)), ((2, -4, 1), (1, 5, 1), (1, 5, 1), (2, -4, 1)),
         ((5, 5, 1), (0, 1, 1), (0, 1, 1), (5, 5, 1))]
MID_N = [((4, 9, 1), (2, -12, 1), (6, -4, 1), (0, 1, 1))]  # reference arithmetic: ~1e-5 relative
HIGH_N = [((7, 3, 1), (6, -4, 1), (6, -4, 1), (7, 3, 1)), ((9, 1, 1), (9, -1, 1), (9, -1, 1), (9, 1, 1))]


@pytest.mark.parametrize("q", LOW_N + MID_N + HIGH_N)
def test_v_int_quad_matches_exact_rational(q):
    from oracle.vint_exact import v_int_exact

    ex = v_int_exact(*q)
    assert qd.v_int(*q, quad=True) == pytest.approx(ex, rel=2e-12, abs=1e-15)


@pytest.mark.parametrize("q", LOW_N)
def test_v_int_reference_arithmetic_low_n(q):
    from oracle.vint_exact import v_int_exact

    assert qd.v_int(*q) == pytest.approx(v_int_exact(*q), rel=1e-9, abs=1e-14)


@pytest.mark.parametrize("q", HIGH_N)
def test_v_int_reference_arithmetic_fails_at_high_n(q):
    # the reference's real(8) accumulation cancels away every digit here;
    # QD_TBME_QUAD exists for this
    from oracle.vint_exact import v_int_exact

    ex = v_int_exact(*q)
    assert abs(qd.v_int(*q) - ex) > 10 * abs(ex)


@pytest.mark.parametrize("nbody,hw,ref", [(2, 1.0, 3.1619), (6, 1.0, 20.7192), (6, 0.28, 8.0196)])
def test_hartree_fock_energy_published(nbody, hw, ref):
    # published HF energies of the 2-D dot (10 shells), e.g. 3.1619 / 20.7192 / 8.0196
    vec, eig, it = qd.hf_hamiltonian(nbody, 10, hw)
    assert abs(vec[0] - ref) < 1e-4
    assert it < 100


def test_hartree_fock_basis_invariants():
    n, R = 6, 8
    vec, eig, it = qd.hf_hamiltonian(n, R, 1.0)
    L = qd.Layout(n, R, eig=eig, device=qd.HOST_ONLY)
    mp = L.msp - n
    fhh = vec[1:1 + n * n].reshape(n, n, order="F")
    fpp = vec[1 + n * n:1 + n * n + mp * mp].reshape(mp, mp, order="F")
    fph = vec[1 + n * n + mp * mp:1 + n * n + mp * mp + mp * n]
    assert np.abs(fph).max() < 1e-8                     # Brillouin: no ph Fock block
    assert np.allclose(np.diag(fhh), eig[:n], atol=1e-10)  # diagonal Fock in the HF basis
    assert np.allclose(np.diag(fpp), eig[n:], atol=1e-10)
    # holes are the N lowest HF states and the layout accepts them
    assert np.all(eig[:n].max() < eig[n:].min())


def test_hartree_fock_deterministic_and_mebin_roundtrip(tmp_path):
    path = os.path.join(tmp_path, "ME.bin")
    qd.tbme_write(6, path, nthreads=3)
    assert os.path.getsize(path) % 40 == 0
    v1, e1, _ = qd.hf_hamiltonian(6, 6, 1.0, nthreads=1)
    v2, e2, _ = qd.hf_hamiltonian(6, 6, 1.0, mebin=path, nthreads=4)
    assert np.array_equal(v1, v2) and np.array_equal(e1, e2)
