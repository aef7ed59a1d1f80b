"""The native library without a GPU: exports, host model build, argument checks."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import os_d_b200 as q
from os_d_b200 import _native as N
from oracle import oracle_py as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "qjx_b200.h")).read()
    return sorted(set(re.findall(r"\b(qjx_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_entry_point():
    lib = C.CDLL(N.LIB_PATH)
    names = header_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) <= set(N.EXPORTS)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(N, "LIB_PATH", str(tmp_path / "absent.so"))
    monkeypatch.setattr(N, "_lib", None)
    with pytest.raises(N.QjxError, match="native library missing"):
        N.lib()


@pytest.mark.parametrize("Nb", [5, 40])
def test_host_model_is_bit_identical_to_oracle(Nb):
    H, Hd, L, Ut = q.build_dimer(Nb, 1.0, 0.5, 1.0, 1.5, 0.1, 1.0, 12)
    H2, Hd2, L2, K0, K1 = O.dimer_operators(Nb, 1.0, 0.5, 1.0, 1.5, 0.1)
    assert np.array_equal(H, H2) and np.array_equal(Hd, Hd2) and np.array_equal(L, L2)
    K = q.dimer_generators(Nb, 1.0, 0.5, 1.0, 1.5, 0.1)
    assert np.array_equal(K[0], K0) and np.array_equal(K[1], K1)
    T = 2.0 * 3.1415926535897932384626433832795
    assert np.array_equal(Ut[0], O.split_tree(K0, T, 12)) and np.array_equal(Ut[1], O.split_tree(K1, T, 12))


def test_expm_matches_oracle():
    rng = np.random.default_rng(2)
    A = (rng.standard_normal((33, 33)) + 1j * rng.standard_normal((33, 33))) * 0.7
    assert np.allclose(q.expm(A), O.expm(A), rtol=0, atol=1e-13 * np.abs(O.expm(A)).max())


def mcg31_leapfrog(seed, k, s, count):
    m, a = 2 ** 31 - 1, 1132489760
    x0 = seed % m or 1
    x = pow(a, k + 1, m) * x0 % m
    step = pow(a, s, m)
    out = []
    for _ in range(count):
        out.append(x / m)
        x = x * step % m
    return out


@pytest.mark.parametrize("rtype", [0, 1, 2])
def test_random_observables(rtype):
    d, num, seed, mns = 7, 2, 100, 1000000
    R = q.random_observables(d, num, seed, mns, rtype)
    for o in range(num):
        u = mcg31_leapfrog(3873247, seed + o, mns, 4 * d * d)
        g = [np.sqrt(-2 * np.log(u[2 * i])) * np.sin(2 * 3.1415926535897932384626433832795 * u[2 * i + 1])
             for i in range(2 * d * d)]
        X = 0.5 * (np.array(g[: d * d]).reshape(d, d) + 1j * np.array(g[d * d:]).reshape(d, d))
        ref = X @ X.conj().T
        if rtype:
            ref = ref / (np.trace(ref).real / (d if rtype == 2 else 1))
        assert np.allclose(R[o], ref, rtol=1e-12, atol=1e-12)
        assert np.allclose(R[o], R[o].conj().T, atol=1e-12)
        assert np.linalg.eigvalsh(R[o]).min() > -1e-12
    if rtype == 2:
        assert np.isclose(np.trace(R[0]).real, d)


def test_create_rejects_bad_arguments_before_touching_a_gpu():
    lib = N.lib()
    d = 5
    U = np.zeros((2, 4, d, d), np.complex128)
    Lm = np.zeros((d, d), np.complex128)
    HE = np.zeros((d, d), np.complex128)
    g = np.ones(1)
    h = C.c_void_p()

    def create(**kw):
        cfg = N.QjxConfig()
        cfg.d, cfg.n_traj, cfg.deep, cfg.num_branches, cfg.num_diss = d, 4, 4, 2, 1
        cfg.T, cfg.max_dumps = 6.28, 1
        for k, v in kw.items():
            setattr(cfg, k, v)
        return lib.qjx_create(C.byref(cfg), N.dp(U), N.dp(Lm), N.dp(g), N.dp(HE), None, C.byref(h))

    assert create(d=1) == 1           # QJX_ERR_INVALID_ARG
    assert create(n_traj=0) == 1
    assert create(T=0.0) == 1
    assert create(num_robs=1) == 1    # R missing
    assert create(d=1025) == 8        # QJX_ERR_UNSUPPORTED: d > 1024
    assert create(d=300, precision=1) == 8  # the split form takes d <= 256
    assert lib.qjx_create(None, None, None, None, None, None, C.byref(h)) == 1


def test_status_strings():
    lib = N.lib()
    assert lib.qjx_status_string(3) == b"norm more than 1"
    assert lib.qjx_status_string(4) == b"injected uniform sequence exhausted"
