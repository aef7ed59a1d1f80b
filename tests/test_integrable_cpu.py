"""The Integrable system (sys_id 5) on the host: the oracle's operators against a numpy
restatement built with np.kron exactly as IntegrableNewDelBehaviour composes them
(newdel.cpp:1924-2076 dissipators, 1030-1095 special matrix, 2914-3004 hamiltonians_qj), the
product builder (qjx_build_integrable) against the oracle bit for bit, and the disorder normals
against a pure-Python MCG31m1 + Box-Muller restatement."""
import numpy as np
import pytest

from oracle import oracle_py as O
from tests.test_native_cpu import mcg31_leapfrog


def numpy_integrable(N, seed, num_seeds, tau, k):
    con = np.zeros((4, 4), complex)
    con[0, 0], con[3, 3], con[1, 2], con[2, 1] = tau, k, 1, 1
    eye = np.eye(2)
    d = 1 << N
    Ls = []
    left = con
    for _ in range(2, N):
        left = np.kron(left, eye)
    Ls.append(left)
    for c in range(1, N - 2):  # middle channels
        m = eye
        for _ in range(1, c):
            m = np.kron(m, eye)
        m = np.kron(m, con)
        for _ in range(c + 2, N):
            m = np.kron(m, eye)
        Ls.append(m)
    right = eye
    for _ in range(1, N - 2):
        right = np.kron(right, eye)
    Ls.append(np.kron(right, con))
    border = np.zeros((d, d), complex)  # con on (spin N-1, spin 0)
    for s in range(d):
        bits = [(s >> (N - 1 - i)) & 1 for i in range(N)]  # most significant first
        if bits[0] == bits[-1]:
            border[s, s] = tau if bits[0] == 0 else k
        else:
            inv = list(bits)
            inv[0], inv[-1] = bits[-1], bits[0]
            border[int("".join(map(str, inv)), 2), s] = 1
    Ls.append(border)
    u = mcg31_leapfrog(13371337, seed, num_seeds, 2 * d * d)
    g = np.array([np.sqrt(-2 * np.log(u[2 * i])) * np.sin(2 * 3.1415926535897932384626433832795 * u[2 * i + 1])
                  for i in range(d * d)]).reshape(d, d)
    X = g + 1j * g
    y = 0.5 * (X + X.conj().T)
    y = y / np.sqrt(np.trace(y @ y).real)
    S = y / np.sqrt(d)
    K = -1j * (-0.5j * sum(L.conj().T @ L for L in Ls))
    return np.stack(Ls), S, K


@pytest.mark.parametrize("N,tau,k", [(3, 1.0, -1.0), (4, 0.3, 0.7), (6, 1.0, -1.0)])
def test_oracle_operators_follow_the_reference_definitions(N, tau, k):
    L, S, K = O.integrable_operators(N, 2, 1000000, tau, k)
    L2, S2, K2 = numpy_integrable(N, 2, 1000000, tau, k)
    assert np.array_equal(L, L2)
    assert np.allclose(S, S2, rtol=0, atol=1e-14) and np.allclose(S, S.conj().T, atol=0)
    assert np.allclose(K, K2, rtol=0, atol=1e-14)
    assert abs(np.trace(S @ S).real * (1 << N) - 1.0) < 1e-12


def test_product_builder_equals_oracle():
    import os_d_b200 as q

    L, S, K = O.integrable_operators(5, 7, 1000000, 1.0, -1.0)
    L2, S2, Ut = q.build_integrable(5, 7, 1000000, 1.0, -1.0, 1.25, 10)
    assert np.array_equal(L, L2) and np.array_equal(S, S2)
    assert np.array_equal(Ut, O.split_tree(K, 1.25, 10))


def test_bad_sizes_rejected():
    import os_d_b200._native as N

    assert N.lib().qjx_build_integrable(2, 1, 1, 1.0, 1.0, 1.0, 4, None, None, None, None) == 1
    assert N.lib().qjx_build_integrable(11, 1, 1, 1.0, 1.0, 1.0, 4, None, None, None, None) == 1


def test_ps_product_builder_equals_oracle():
    """PS (sys_id 2): qjx_build_ps against orc_ps_operators bit for bit, and the oracle against a
    numpy Kronecker restatement of PSNewDelBehaviour (newdel.cpp:650-866, 1582-1697, 2603-2749)."""
    import os_d_b200 as q

    ns, nps, al, dp, gp, A, w = 2, 6, 5.0, 1.3, 0.7, 3.2, 0.05
    H, Hd, L, S, K0, K1 = O.ps_operators(ns, nps, al, dp, gp, A, 1, w)
    H2, Hd2, L2, S2, Ut = q.build_ps(ns, nps, al, dp, gp, A, 1, w, 0.5, 1.5, 8)
    assert all(np.array_equal(x, y) for x, y in ((H, H2), (Hd, Hd2), (L, L2), (S, S2)))
    assert np.array_equal(Ut[0], O.split_tree(K0, 0.5 * al, 8)) and np.array_equal(Ut[1], O.split_tree(K1, 1.5 * al, 8))
    a = np.diag(np.sqrt(np.arange(1, nps)), 1)
    sz, sm, sp, I2 = np.diag([1.0, -1.0]), np.array([[0, 0], [1, 0.0]]), np.array([[0, 1], [0, 0.0]]), np.eye(2)

    def spin_op(sig, s):
        m = sig if s == 0 else I2
        for it in range(1, ns):
            m = np.kron(m, sig if it == s else I2)
        return m

    Jz, Jm, Jp = (0.5 * sum(spin_op(sig, s) for s in range(ns)) for sig in (sz, sm, sp))
    Is, Ip = np.eye(1 << ns), np.eye(nps)
    Hn = (np.kron(dp * 0.5 * Jz, Ip) + gp * 0.5 * (np.kron(Is, a.T) @ np.kron(Jm, Ip) + np.kron(Jp, Ip) @ np.kron(Is, a))
          + np.kron(Is, 0.5 / al ** 3 * a.T @ a.T @ a @ a))
    assert np.allclose(H, Hn, rtol=0, atol=1e-15)
    Ls = [np.kron(Is, a)] + [np.kron(spin_op(sm, s), Ip) for s in range(ns)]
    assert np.array_equal(L, np.array(Ls, complex))
    for got, want in zip(S, (np.kron(Is, a), np.kron(Jz, Ip), np.kron(Jp, Ip), np.kron(Is, a.T @ a))):
        assert np.array_equal(got, want.astype(complex))
    He = Hn - 0.5j * sum(g * Lc.T @ Lc for g, Lc in zip([1 / (4 * al)] + [w] * ns, Ls))
    assert np.allclose(K0, -1j * He + A * np.kron(Is, a.T - a), atol=1e-14)
    assert np.allclose(K1, -1j * He, atol=1e-14)
