"""The f-basis Liouvillian and RK4 against the reference's own code.

oracle/_ref/libfbref.so is the unmodified source/cpp/CQdiss_os_dimer solver (CQdiss, SparceM_op,
read_config) built by oracle/build_ref.py against a shim of the four MKL routines it calls.  These
tests pin the oracle's dense projection (oracle/fbasis_oracle.c), the library's banded builder
(qjx_fb_build_dimer) and the oracle's RK4 to what the reference assembles and integrates:
f_basis_init (CQdiss/f_basis_init.cpp:11-104) and calcODE_trans (CQdiss/calcODE.cpp:249-309).
Skipped where the reference tree was not available to build the library.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle_py as O

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libfbref.so")

pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="reference f-basis library not built here")

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)


def _lib():
    L = C.CDLL(LIB)
    L.fbref_build.argtypes = [C.c_int] + [C.c_double] * 4 + [C.c_int, ip, ip, ip, ip, dp, ip, ip, dp, dp, dp, dp]
    L.fbref_rk4.argtypes = [C.c_int] + [C.c_double] * 4 + [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, dp]
    return L


def _p(a, t):
    return a.ctypes.data_as(t)


def ref_build(N, J, U, E, g, start=0):
    """Gs, Qs_drv (scipy CSR), Ks and the initial f-vector as the reference assembles them."""
    import scipy.sparse as sp

    L = _lib()
    gn, qn = C.c_int(), C.c_int()
    assert L.fbref_build(N, J, U, E, g, start, C.byref(gn), C.byref(qn), None, None, None, None, None, None, None,
                         None, None) == 0
    n = (N + 1) ** 2 - 1
    gr, gc, gv = np.zeros(n + 1, np.int32), np.zeros(gn.value, np.int32), np.zeros(gn.value)
    qr, qc, qv = np.zeros(n + 1, np.int32), np.zeros(qn.value, np.int32), np.zeros(qn.value)
    ks, x0, mi = np.zeros(n), np.zeros(n), C.c_double()
    assert L.fbref_build(N, J, U, E, g, start, C.byref(gn), C.byref(qn), _p(gr, ip), _p(gc, ip), _p(gv, dp),
                         _p(qr, ip), _p(qc, ip), _p(qv, dp), _p(ks, dp), _p(x0, dp), C.byref(mi)) == 0
    return (sp.csr_matrix((gv, gc, gr), shape=(n, n)), sp.csr_matrix((qv, qc, qr), shape=(n, n)), ks, x0,
            mi.value)


def antisym_sign(N):
    """+1 on the symmetric and diagonal coordinates, -1 on the antisymmetric ones (the f-index layout
    of initRhoODE: pairs (sym, antisym) for i < j, then the N diagonal coordinates)."""
    d = N + 1
    s = np.ones(d * d - 1)
    s[1 : d * (d - 1) : 2] = -1.0
    return s


def builder(N, J, U, E, g):
    import scipy.sparse as sp

    from os_d_b200 import _native as Nt

    (gr, gc, gv), (qr, qc, qv), kb = Nt.fb_build_dimer(N, J, U, E, g)
    n = kb.size
    return sp.csr_matrix((gv, gc, gr), shape=(n, n)), sp.csr_matrix((qv, qc, qr), shape=(n, n)), kb


# The reference's coherent part has the opposite sign convention on the antisymmetric coordinates:
# its generator equals S G S with S = diag(antisym_sign), i.e. it evolves the complex conjugate
# rho*, which has the same populations (H and L are real).  Everything below compares S G S.


@pytest.mark.parametrize("N,J,U,E", [(2, 1.0, 0.5, 1.0), (5, 0.7, 1.3, -0.4), (15, 1.0, 0.5, 1.0), (50, 1.0, 0.5, 1.0)])
def test_reference_hamiltonian_and_drive_equal_builder(N, J, U, E):
    """No dissipation: Gs = Qs_base and Qs_drv (CalcQs.cpp:141-173) equal the library's builder and the
    oracle's projection, up to the antisymmetric sign convention, to 1e-13 of the largest entry."""
    import scipy.sparse as sp

    Gr, Qr, Kr, _, max_imag = ref_build(N, J, U, E, 0.0)
    assert max_imag < 1e-15  # rounding residue of complex arithmetic on a real problem
    Gb, Qb, Kb = builder(N, J, U, E, 0.0)
    S = sp.diags(antisym_sign(N))
    scale = abs(Gr).max()
    assert abs(S @ Gb @ S - Gr).max() <= 1e-13 * scale
    assert abs(S @ Qb @ S - Qr).max() <= 1e-13 * abs(Qr).max()
    assert np.abs(Kb - Kr).max() <= 1e-15
    if N <= 15:
        Go, Qo, Ko = O.fb_dense(N, J, U, E, 0.0)
        assert np.abs(S @ Go @ S - Gr.toarray()).max() <= 1e-13 * scale


@pytest.mark.parametrize("N,J,U,E,g", [(1, 1.0, 0.5, 1.0, 0.1), (2, 1.0, 0.5, 1.0, 0.1), (5, 1.0, 0.5, 1.0, 0.1),
                                       (6, 0.7, 1.3, -0.4, 0.3), (10, 1.0, 0.5, 1.0, 0.1), (20, 1.0, 0.5, 1.0, 0.1)])
def test_reference_liouvillian_equals_builder_and_oracle(N, J, U, E, g):
    """The whole Liouvillian Gs = Qs_base + Rs (calcRs_dimer, CalcRs.cpp:385-468; calc_Gs) and Ks
    (calcKs_dimer) against the builder and the oracle's dense projection."""
    import scipy.sparse as sp

    Gr, Qr, Kr, _, max_imag = ref_build(N, J, U, E, g)
    assert max_imag < 1e-15
    Gb, Qb, Kb = builder(N, J, U, E, g)
    Go, Qo, Ko = O.fb_dense(N, J, U, E, g)
    S = sp.diags(antisym_sign(N))
    scale = abs(Gr).max()
    assert abs(S @ Gb @ S - Gr).max() <= 1e-13 * scale
    assert np.abs(S @ Go @ S - Gr.toarray()).max() <= 1e-13 * scale
    big = 1e-12 * scale  # the same structural nonzeros (the reference keeps explicit zeros of its sums)
    assert np.array_equal(np.abs(Gr.toarray()) > big, np.abs(Go) > big)
    assert np.abs(Kb - Kr).max() <= 1e-13 * max(np.abs(Kr).max(), 1.0)
    assert np.abs(Ko - Kr).max() <= 1e-13 * max(np.abs(Kr).max(), 1.0)


@pytest.mark.parametrize("N,bad_rows", [(3, 3), (15, 3)])
def test_reference_dissipator_defect_is_confined_to_a_few_rows(N, bad_rows):
    """At some sizes (N = 3, 7, 15 and 50 among those checked) the reference's dissipator, which its
    own tensor code assembles without any MKL call (calcRs_dimer), differs from the Lindblad form in
    a few rows: there it couples symmetric and antisymmetric coordinates, which a real jump operator
    cannot do.  The builder and the oracle keep the exact projection of the Lindblad dissipator; this
    test records where the reference departs from it."""
    import scipy.sparse as sp

    Gr, _, _, _, _ = ref_build(N, 0.0, 0.0, 0.0, 0.1)
    Gb, _, _ = builder(N, 0.0, 0.0, 0.0, 0.1)
    s = antisym_sign(N)
    S = sp.diags(s)
    R, B = Gr.toarray(), (S @ Gb @ S).toarray()
    bad = np.abs(R - B) > 1e-9 * np.abs(R).max()
    assert len(set(np.nonzero(bad)[0])) == bad_rows
    # a real jump operator: the exact dissipator never mixes symmetric (incl. diagonal) and
    # antisymmetric coordinates; the reference's deviating rows do
    mix = np.not_equal.outer(s > 0, s > 0)
    assert np.abs(B[mix]).max() < 1e-13
    assert np.abs(R[mix]).max() > 1e-2


@pytest.mark.parametrize("N,k", [(3, 0), (7, 2), (12, 12)])
def test_reference_initial_vector_equals_oracle(N, k):
    import os_d_b200 as q

    _, _, _, x0, _ = ref_build(N, 1.0, 0.5, 1.0, 0.1, start=k)
    rho = np.zeros((N + 1, N + 1), complex)
    rho[k, k] = 1
    assert np.abs(O.fb_x_from_rho(N, rho) - x0).max() < 1e-15
    assert np.abs(q.fbasis_pure_state(N, k) - x0).max() < 1e-15


@pytest.mark.parametrize("N,drv_type,periods", [(4, 0, 2), (6, 1, 1), (10, 0, 1)])
def test_reference_rk4_equals_oracle_rk4(N, drv_type, periods):
    """The reference's calcODE_trans (2 pi periods of num_steps RK4 steps, sign or sine drive, CSR
    products with mkl_dcsrgemv's semantics) against the oracle's RK4 from |0><0|: equal to rounding,
    with the antisymmetric coordinates of opposite sign."""
    J, U, E, g, A, steps = 1.0, 0.5, 1.0, 0.1, 1.5, 300
    n = (N + 1) ** 2 - 1
    x_ref = np.zeros(n)
    assert _lib().fbref_rk4(N, J, U, E, g, drv_type, A, steps, periods, 0, _p(x_ref, dp)) == 0
    Go, Qo, Ko = O.fb_dense(N, J, U, E, g)
    rho0 = np.zeros((N + 1, N + 1), complex)
    rho0[0, 0] = 1
    x_o = O.fb_rk4(O.fb_csr(Go), O.fb_csr(Qo), Ko, O.fb_x_from_rho(N, rho0), A, drv_type=drv_type, T=2 * np.pi,
                   num_steps=steps, n_periods=periods)
    assert np.abs(x_o - O.fb_x_from_rho(N, rho0)).max() > 1e-3  # the state moved
    assert np.abs(antisym_sign(N) * x_o - x_ref).max() < 1e-12
    # populations (the diagonal of rho) are the same in both conventions
    assert np.allclose(np.diag(O.fb_rho(N, x_o)).real, np.diag(O.fb_rho(N, x_ref)).real, atol=1e-12)
