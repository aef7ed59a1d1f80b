"""The oracle's RK propagator (prop_id 1: RK4 of the non-Hermitian Schroedinger equation with
linear interpolation of the jump time, source/cpp/QJX/QJX/core.cpp:11886-11948) against
independent answers: the exact propagator without dissipation, the f-basis Lindblad density
matrix with dissipation, and the interpolation property of the recorded jumps."""
import numpy as np
import pytest
import scipy.linalg as sl

from oracle import oracle_py as O
from tests.helpers import T2PI


def rk_problem(N, J=1.0, U=0.5, E=1.0, A=1.5, g=0.1):
    H, Hd, L, K0, K1 = O.dimer_operators(N, J, U, E, A, g)
    gamma = g / N
    Heff = H - 0.5j * gamma * (L.conj().T @ L)
    return H, Hd, L, Heff


def rk_ensemble(N, n, Heff, L, HE, seed=3, record=2):
    d = N + 1
    dummy_U = np.zeros((2, 1, d, d), complex)
    ens = O.Ensemble(dummy_U, L, [1.0], HE, None, T2PI, n, seed=seed, record=record, rec_cap=4096)
    ens.init(0, 0)
    return ens


def test_rk_without_dissipation_matches_exact_propagator():
    N, E0 = 8, 1.0
    H, Hd, L, Heff = rk_problem(N, A=0.0, g=0.0)
    psi0 = np.zeros(N + 1, complex)
    psi0[0] = 1
    exact = sl.expm(-1j * (H + E0 * Hd) * T2PI) @ psi0
    errs = []
    for rk_ns in (2000, 4000):
        ens = rk_ensemble(N, 4, Heff, L, H + E0 * Hd)
        assert ens.run_periods_rk(1, Heff, Hd, E0, 0.0, rk_ns=rk_ns) == 0
        assert ens.jumps_counts.sum() == 0
        assert np.allclose(ens.t, T2PI, rtol=0, atol=1e-12)
        errs.append(np.abs(ens.phi - exact).max())
    assert errs[1] < 1e-6
    assert 12 < errs[0] / errs[1] < 20  # fourth order


def test_rk_jumps_are_interpolated_to_the_threshold():
    N = 10
    H, Hd, L, Heff = rk_problem(N, g=1.0)
    ens = rk_ensemble(N, 16, Heff, L, H + Hd)
    rk_ns = 500
    assert ens.run_periods_rk(2, Heff, Hd, 1.0, 1.5, rk_ns=rk_ns) == 0
    assert ens.jumps_counts.sum() > 20
    h = T2PI / rk_ns
    for tr in range(ens.n):
        t, ty, nrm, eta = ens.jumps(tr)
        assert np.all(np.diff(t) >= 0) and np.all((t > 0) & (t < 2 * T2PI + 1e-9))
        assert np.all(ty == 0)
        # the begin part lands near the threshold: the norm is interpolated linearly inside the
        # step, and the reference's stage arguments always use the full step (arg_upd)
        assert np.all(np.abs(nrm - eta) < 0.05), np.abs(nrm - eta).max()
        assert np.median(np.abs(nrm - eta)) < 10 * h, np.median(np.abs(nrm - eta))


def test_rk_ensemble_within_statistical_error_of_fbasis_rho():
    N, n, periods = 4, 3000, 2
    J, U, E, A, g = 1.0, 0.5, 1.0, 1.5, 2.0
    H, Hd, L, Heff = rk_problem(N, J, U, E, A, g)
    Gs, Qs, Ks = O.fb_dense(N, J, U, E, g)
    rho0 = np.zeros((N + 1, N + 1), complex)
    rho0[0, 0] = 1
    x = O.fb_rk4(O.fb_csr(Gs), O.fb_csr(Qs), Ks, O.fb_x_from_rho(N, rho0), A, T=T2PI, num_steps=2000,
                 n_periods=periods)
    pops_f = np.real(np.diag(O.fb_rho(N, x)))
    ens = rk_ensemble(N, n, Heff, L, H + E * Hd, seed=17, record=0)
    assert ens.run_periods_rk(periods, Heff, Hd, E, A, rk_ns=400) == 0
    adr = ens.observables(want_adr=True)["adr"]
    err = adr.std(axis=0) / np.sqrt(n)
    assert np.all(np.abs(adr.mean(axis=0) - pops_f) < 4.5 * err + 2e-3), (adr.mean(axis=0), pops_f)


@pytest.mark.parametrize("N", [5, 100])
def test_library_rk_operators_equal_oracle(N):
    import os_d_b200 as q

    He, Hd = q.build_dimer_rk(N, 1.0, 0.5, 1.0, 0.1)
    assert np.array_equal(He, O.dimer_heff(N, 1.0, 0.5, 1.0, 0.1))
    assert np.array_equal(Hd, O.dimer_operators(N, 1.0, 0.5, 1.0, 1.5, 0.1)[1])
