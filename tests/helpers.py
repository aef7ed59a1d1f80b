"""Shared problem builders for the tests (oracle side and engine side)."""
import numpy as np

from oracle import oracle_py as O

T2PI = 2.0 * 3.1415926535897932384626433832795


def dimer_problem(N, J=1.0, U=0.5, E=1.0, A=1.5, g=0.1, omega=1.0, deep=16):
    """Operators and split tree of the driven dissipative dimer, built by the oracle."""
    H, Hd, L, K0, K1 = O.dimer_operators(N, J, U, E, A, g)
    T = T2PI / omega
    Ut = np.stack([O.split_tree(K0, T, deep), O.split_tree(K1, T, deep)])
    HE = H + E * Hd
    return dict(H=H, Hd=Hd, L=L, U=Ut, HE=HE, T=T, d=N + 1, deep=deep)


def random_observable(d, seed):
    """A Hermitian positive observable X X^H / (tr / d) (the random_obs_type 2 form, newdel.cpp:3699-3741)."""
    rng = np.random.default_rng(seed)
    X = 0.5 * (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d)))
    R = X @ X.conj().T
    return R / (np.trace(R).real / d)


def start_states(n, d, start_type=0, start_state=0):
    psi = np.zeros((n, d), np.complex128)
    if start_type == 0:
        psi[:, start_state] = 1.0
    else:
        psi[:] = np.sqrt(1.0 / d)
    return psi
