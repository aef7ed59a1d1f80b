"""Ensemble purity Tr(rho^2) of the trajectory ensemble (rho = (1/n) sum |psi_hat><psi_hat|).

QJX computes no ensemble purity; the formula is calc_purity's
(source/cpp/CQdiss/CQdiss/CalcTraseRO2.cpp:57-75), whose f-basis form is 1/(N+1) + ||x||^2.
"""
import numpy as np
import pytest

from oracle import oracle_py as O
from tests.helpers import T2PI, dimer_problem, start_states


def test_oracle_purity_matches_numpy_on_random_states():
    rng = np.random.default_rng(3)
    psi = rng.normal(size=(37, 9)) + 1j * rng.normal(size=(37, 9))
    p, rho = O.purity(psi)
    hat = psi / np.linalg.norm(psi, axis=1, keepdims=True)
    ref = hat.T @ hat.conj() / len(psi)
    assert np.abs(rho - ref).max() < 1e-15
    assert abs(p - np.sum(np.abs(ref) ** 2)) < 1e-14
    assert abs(np.trace(rho).real - 1) < 1e-14


def test_oracle_purity_limits():
    d = 6
    same = np.tile(np.exp(1j * np.arange(d)) * (np.arange(d) + 1.0), (5, 1))
    assert abs(O.purity(same)[0] - 1) < 1e-15  # identical states: pure ensemble
    basis = np.eye(d, dtype=complex) * 3.0
    assert abs(O.purity(basis)[0] - 1.0 / d) < 1e-16  # orthogonal states: maximally mixed


def test_ensemble_purity_estimates_fbasis_purity():
    """E[purity of n sampled pure states] = 1/n + (1 - 1/n) Tr rho^2 for the Lindblad rho."""
    N, n = 4, 3000
    J, U, E, A, g = 1.0, 0.5, 1.0, 1.5, 2.0
    Gs, Qs, Ks = O.fb_dense(N, J, U, E, g)
    rho0 = np.zeros((N + 1, N + 1), complex)
    rho0[0, 0] = 1
    x = O.fb_rk4(O.fb_csr(Gs), O.fb_csr(Qs), Ks, O.fb_x_from_rho(N, rho0), A, T=T2PI, num_steps=2000, n_periods=2)
    pur_f = 1.0 / (N + 1) + float(x @ x)
    r = O.fb_rho(N, x)
    assert abs(pur_f - np.sum(np.abs(r) ** 2)) < 1e-12  # f-basis form of Tr rho^2
    H, Hd, L, K0, K1 = O.dimer_operators(N, J, U, E, A, g)
    Ut = np.stack([O.split_tree(K0, T2PI, 16), O.split_tree(K1, T2PI, 16)])
    ens = O.Ensemble(Ut, L, [1.0], H + E * Hd, None, T2PI, n, seed=5, record=0)
    ens.init(0, 0)
    assert ens.run_periods(2) == 0
    p_ens, _ = O.purity(ens.phi)
    expect = 1.0 / n + (1 - 1.0 / n) * pur_f
    assert 0.2 < pur_f < 0.99
    assert abs(p_ens - expect) < 0.02, (p_ens, expect)


@pytest.mark.gpu
@pytest.mark.parametrize("N,n", [(20, 64), (200, 300)])
def test_gpu_purity_bit_exact(N, n):
    import os_d_b200 as q

    P = dimer_problem(N)
    eng = q.Engine(P["U"], P["L"], [1.0], P["HE"], None, P["T"], n, seed=11, record=0)
    eng.set_states(start_states(n, P["d"], 0, 0))
    eng.init_thresholds()
    assert eng.purity() == 1.0  # all trajectories in |N,0>
    eng.run_periods(2)
    p_g, rho_g = eng.purity(want_rho=True)
    psi = eng.states()[0]
    p_o, rho_o = O.purity(psi)
    assert np.array_equal(rho_g, rho_o)
    assert p_g == p_o
    assert 0.0 < p_g < 1.0
