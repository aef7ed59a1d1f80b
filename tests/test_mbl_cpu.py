"""The MBL system (sys_id 3) on the host: the oracle's operators against a direct numpy
restatement of MBLNewDelBehaviour (newdel.cpp:182-271 basis, 868-958 H, 1699-1815 dissipators,
2751-2838 hamiltonians_qj), the product builder (qjx_build_mbl) against the oracle bit for bit,
the disorder stream against a pure-Python MCG31m1 leapfrog, and the imbalance
(get_imbalance_mbl, experiment.cpp:1753-1800) of the product against the oracle's."""
import math

import numpy as np
import pytest

from oracle import oracle_py as O
from tests.test_native_cpu import mcg31_leapfrog


def numpy_mbl(Nc, W, U, J, energies, diss_type, phi, gamma):
    """H, L, K from the reference's definitions, written independently of both C builders."""
    xs = [x for x in range(1 << Nc) if bin(x).count("1") == Nc // 2]
    d = len(xs)

    def vb(x):  # convert_int_to_vector_of_bits: most significant cell first
        return [(x >> (Nc - 1 - c)) & 1 for c in range(Nc)]

    def adj(g):
        return bin(g).count("1") == 2 and bin(g & (g << 1)).count("1") == 1

    H = np.zeros((d, d), complex)
    for s, x in enumerate(xs):
        H[s, s] += W * sum(b * e for b, e in zip(vb(x), energies)) + U * bin(x & (x << 1)).count("1")
    for s, x in enumerate(xs):
        for t, y in enumerate(xs):
            H[s, t] -= J * adj(x ^ y)
    nd = Nc if diss_type == 0 else Nc - 1
    L = np.zeros((nd, d, d), complex)
    for c in range(nd):
        for s, x in enumerate(xs):
            bit = lambda v, p: (v >> p) & 1  # noqa: E731  bit_at
            L[c, s, s] = bit(x, c) if diss_type == 0 else bit(x, c) - bit(x, c + 1)
            if diss_type == 1 and bit(x, c) != bit(x, c + 1):
                for t, y in enumerate(xs):
                    g = x ^ y
                    if adj(g):
                        hop = sorted([(Nc - 1) - c2 for c2 in range(Nc) if vb(g)[c2]], reverse=True)
                        if hop[1] == c:
                            L[c, s, t] = -np.exp(-1j * phi) if bit(x, c) else np.exp(1j * phi)
    Heff = H - 0.5j * gamma * sum(Lc.conj().T @ Lc for Lc in L)
    return np.array(xs), H, L, -1j * Heff


@pytest.mark.parametrize("Nc,diss_type", [(4, 0), (6, 1), (8, 1), (8, 0)])
def test_oracle_operators_follow_the_reference_definitions(Nc, diss_type):
    W, U, J, seed, mns, phi, gamma = 3.0, 1.0, 1.0, 5, 1000000, 0.4, 0.1
    xs = O.mbl_basis(Nc)
    assert len(xs) == math.comb(Nc, Nc // 2)
    en, H, L, K = O.mbl_operators(Nc, W, U, J, seed, mns, diss_type, phi, gamma)
    u = mcg31_leapfrog(77778888, seed, mns, Nc)
    assert np.array_equal(en, -1.0 + 2.0 * np.array(u))
    xs2, H2, L2, K2 = numpy_mbl(Nc, W, U, J, en, diss_type, phi, gamma)
    assert np.array_equal(xs, xs2)
    assert np.allclose(H, H2, rtol=0, atol=1e-14) and np.array_equal(H, H.conj().T)
    assert np.allclose(L, L2, rtol=0, atol=1e-15)
    assert np.allclose(K, K2, rtol=0, atol=1e-13)
    if diss_type == 1:  # the hop part makes the channels non-Hermitian
        assert not np.allclose(L[0], L[0].conj().T)


@pytest.mark.parametrize("Nc,diss_type", [(6, 0), (8, 1)])
def test_product_builder_equals_oracle(Nc, diss_type):
    import os_d_b200 as q

    W, U, J, seed, mns, phi, gamma, T, deep = 2.5, 0.7, 1.0, 11, 1000000, 0.25, 0.2, 1.5, 10
    en, H, L, K = O.mbl_operators(Nc, W, U, J, seed, mns, diss_type, phi, gamma)
    en2, xs2, H2, L2, Ut = q.build_mbl(Nc, W, U, J, seed, mns, diss_type, phi, gamma, T, deep)
    assert np.array_equal(en, en2) and np.array_equal(O.mbl_basis(Nc), xs2)
    assert np.array_equal(H, H2) and np.array_equal(L, L2)
    assert np.array_equal(Ut, O.split_tree(K, T, deep))


def test_imbalance_product_equals_oracle():
    import os_d_b200 as q

    Nc = 8
    d = math.comb(Nc, Nc // 2)
    rng = np.random.default_rng(3)
    adr = rng.random((7, d))
    adr /= adr.sum(axis=1, keepdims=True)
    a = q.mbl_imbalance(Nc, adr)
    assert np.array_equal(a, O.mbl_imbalance(Nc, adr))
    # the Neel word 10101010 alone has imbalance +1 (even cells, counted from the most significant)
    xs = O.mbl_basis(Nc)
    one = np.zeros((1, d))
    one[0, list(xs).index(0b10101010)] = 1.0
    assert O.mbl_imbalance(Nc, one)[0] == 1.0


def test_bad_sizes_rejected():
    import ctypes as C

    import os_d_b200._native as N

    d, nd = C.c_int(), C.c_int()
    assert N.lib().qjx_mbl_size(7, 0, C.byref(d), C.byref(nd)) == 1
    assert N.lib().qjx_mbl_size(8, 2, C.byref(d), C.byref(nd)) == 1
    assert N.lib().qjx_mbl_size(12, 1, C.byref(d), C.byref(nd)) == 0 and (d.value, nd.value) == (924, 11)


@pytest.mark.parametrize("lpn_type", [-1, -2, 0])
def test_oracle_mbl_lyapunov_characteristics(lpn_type):
    """MBL LpnMult characteristics (calc_chars_lpn / calc_delta_s, core.cpp:4729-4901) of the oracle
    against numpy on its own states: spec = <psi|H|psi> / (|psi|^2 W), the imbalance of the adr row,
    and delta_s after the perturbation bisection."""
    import os_d_b200 as q

    Nc, W = 8, 2.5
    en, H, L, K = O.mbl_operators(Nc, W, 1.0, 1.0, 3, 1000000, 1, 0.0, 0.1)
    T, deep, n = 10.0, 12, 8
    Ut = O.split_tree(K, T, deep)
    R = q.random_observables(70, 1, 100, 1000000, 2)
    Rs = np.concatenate([H[None], R])
    ens = O.Ensemble(np.stack([Ut, Ut]), L, [1.0] * L.shape[0], H, Rs, T, n, seed=3, record=0, rec_cap=16)
    ens.init(0, 5)
    assert ens.run_periods(1, tr1=n // 2) == 0
    lp = O.Lpn(ens, lpn_type=lpn_type, delta_s=1e-3, mbl_Nc=Nc, spec_div=W)
    lp.start()
    v = lp.values()
    psi = ens.phi
    nrm = np.sum(np.abs(psi) ** 2, axis=1)
    spec = np.einsum("ti,ij,tj->t", psi.conj(), H, psi) / nrm / W
    adr = np.abs(psi) ** 2 / nrm[:, None]
    imb = O.mbl_imbalance(Nc, adr)
    assert np.allclose(v["mean_lpn"], imb, rtol=0, atol=1e-14)
    assert np.allclose(v["robs_lpn"][:, 0] / W, spec, rtol=0, atol=1e-13)
    assert np.allclose(v["robs_lpn"][:, 1], np.einsum("ti,ij,tj->t", psi.conj(), R[0], psi) / nrm, atol=1e-13)
    b, w = np.arange(n // 2), np.arange(n // 2, n)
    if lpn_type == -1:
        ds = np.abs(spec[b] - spec[w])
    elif lpn_type == -2:
        ds = np.abs(imb[w] - imb[b])
    else:
        z = v["robs_lpn"][:, 1]
        ds = np.abs(z[b] - z[w])
    assert np.allclose(v["delta_s"][w], ds, rtol=1e-9, atol=0)
    assert np.allclose(v["delta_s"][w], 1e-3, rtol=1e-6)  # the bisection met the target
