"""A generic QJX system beyond the dimer (num_ham_qj 3 branches, num_diss 3 jump channels with
different rates): the engine takes any propagator tree and jump operators, and the channel
choice of recovery (experiment.cpp:1301-1369) then runs its multi-channel path (channel weights,
cumulative walk, L_idx psi_hat / sqrt(w/g)).  GPU against the oracle, bit for bit."""
import numpy as np
import pytest
import scipy.linalg as sl

from oracle import oracle_py as O
from tests.helpers import T2PI, random_observable, start_states

pytestmark = pytest.mark.gpu


def generic_system(d, seed=4):
    rng = np.random.default_rng(seed)
    H = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
    H = 0.3 * (H + H.conj().T)
    Hd = np.diag(np.linspace(-1.0, 1.0, d)).astype(complex)
    Ls, gs = [], [1.0, 0.5, 2.0]
    for i in range(3):
        M = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
        Ls.append(0.15 * M / np.sqrt(d))
    Heff = H - 0.5j * sum(g * L.conj().T @ L for g, L in zip(gs, Ls))
    Es = [1.5, -0.5, 0.7]  # three branches (num_ham_qj 3)
    deep = 12
    Ut = np.stack([O.split_tree(-1j * (Heff + E * Hd), T2PI * 2.0 / 3.0, deep) for E in Es])
    return Ut, np.stack(Ls), gs, H + Hd


def test_three_branches_three_channels_bit_exact():
    import os_d_b200 as q

    d, n, periods = 24, 48, 2
    Ut, L, gs, HE = generic_system(d)
    R = random_observable(d, 3)[None]
    ens = O.Ensemble(Ut, L, gs, HE, R, T2PI * 2.0 / 3.0, n, seed=13, record=2, rec_cap=20000)
    ens.init(0, 0)
    eng = q.Engine(Ut, L, gs, HE, R, T2PI * 2.0 / 3.0, n, seed=13, record=2, rec_cap=64, keep_adr=1, max_dumps=2)
    eng.set_states(start_states(n, d))
    eng.init_thresholds()
    eng.observe(0, is_start=True)
    o0 = ens.observables(is_start=True, want_adr=True)
    assert ens.run_periods(periods) == 0
    eng.run_periods(periods, dump_at=[periods], dump_base=1)
    o1 = ens.observables(want_adr=True)
    psi, t, eta, jc = eng.states()
    assert jc.sum() > 20
    assert np.array_equal(psi, ens.phi) and np.array_equal(t, ens.t) and np.array_equal(eta, ens.eta)
    types = []
    for tr in range(n):
        for a, b in zip(eng.jumps(tr), ens.jumps(tr)):
            assert np.array_equal(a, b), tr
        types.extend(eng.jumps(tr)[1])
    assert len(set(types)) == 3  # every channel was chosen
    for o, dmp in ((o0, 0), (o1, 1)):
        g = eng.observables(dmp, 1, want_adr=True)
        for k in ("norm", "mean", "dispersion", "m2", "energy"):
            assert np.array_equal(g[k][0], o[k]), k
        assert np.array_equal(g["random_obs"][0], o["random_obs"])


def lindblad_basis_system(d, seed=5, alpha=1.0):
    """A random Lindbladian with num_diss = d^2 - 1 jump channels, the LndHam construction
    (newdel.cpp:958-1029, 1814-1923, 2844-2912): L_k = sqrt(lambda_k) sum_j v_jk F_{j+1} over the
    normalised generalised Gell-Mann basis F, (lambda, v) the eigenpairs of a random G = X X^H with
    trace d, and H a random Hermitian matrix of unit Frobenius norm times alpha / sqrt(d)."""
    rng = np.random.default_rng(seed)
    F = []
    for i in range(d):
        for j in range(i + 1, d):
            A = np.zeros((d, d), complex)
            A[i, j] = A[j, i] = 1 / np.sqrt(2)
            F.append(A)
            B = np.zeros((d, d), complex)
            B[i, j], B[j, i] = -1j / np.sqrt(2), 1j / np.sqrt(2)
            F.append(B)
    for i in range(d - 1):
        Dg = np.zeros((d, d), complex)
        for j in range(i + 1):
            Dg[j, j] = 1 / np.sqrt((i + 1) * (i + 2))
        Dg[i + 1, i + 1] = -(i + 1) / np.sqrt((i + 1) * (i + 2))
        F.append(Dg)
    M = d * d - 1
    X = 0.5 * (rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M)))
    G = X @ X.conj().T
    G = d * G / np.trace(G).real
    lam, V = np.linalg.eigh(G)
    Fs = np.stack(F)
    L = np.stack([np.sqrt(max(lam[k], 0.0)) * np.tensordot(V[:, k], Fs, axes=1) for k in range(M)])
    Y = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
    Y = 0.5 * (Y + Y.conj().T)
    H = alpha / np.sqrt(d) * Y / np.sqrt(np.trace(Y @ Y).real)
    Heff = H - 0.5j * sum(Lk.conj().T @ Lk for Lk in L)
    return H, L, Heff


def test_lindblad_basis_channels_bit_exact():
    """d^2 - 1 = 288 jump channels (more groups than an engine's shared-memory tables could hold):
    every jump computes 288 channel weights, one micro-step each, before the choice."""
    import os_d_b200 as q

    d, n, deep = 17, 24, 10
    H, L, Heff = lindblad_basis_system(d)
    Tb = 2.0  # one branch of length Tb / 2 = 1 per period
    Ut = O.split_tree(-1j * Heff, Tb, deep)[None]
    gs = np.ones(L.shape[0])
    ens = O.Ensemble(Ut, L, gs, H, None, Tb, n, seed=3, record=2, rec_cap=20000)
    ens.init(1, 0)
    eng = q.Engine(Ut, L, gs, H, None, Tb, n, seed=3, record=2, rec_cap=64, max_dumps=1)
    eng.set_states(start_states(n, d, 1))
    eng.init_thresholds()
    assert ens.run_periods(3) == 0
    eng.run_periods(3)
    psi, t, eta, jc = eng.states()
    assert jc.sum() > 10
    assert np.array_equal(psi, ens.phi) and np.array_equal(t, ens.t) and np.array_equal(eta, ens.eta)
    types = []
    for tr in range(n):
        for a, b in zip(eng.jumps(tr), ens.jumps(tr)):
            assert np.array_equal(a, b), tr
        types.extend(eng.jumps(tr)[1])
    assert len(set(types)) > 5


def test_unequal_branch_durations_bit_exact():
    """Branches of different durations in one period (the JCS kick and free evolution,
    init_split_structure_jcs, core.cpp:10086-10124): per-branch split-level steps."""
    import os_d_b200 as q

    d, n, deep = 16, 40, 12
    rng = np.random.default_rng(8)
    H = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
    H = 0.2 * (H + H.conj().T)
    Hd = np.diag(np.linspace(-1.0, 1.0, d)).astype(complex)
    L = (0.2 * (rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))) / np.sqrt(d))[None]
    Heff = H - 0.5j * L[0].conj().T @ L[0]
    lens = np.array([0.35, 2.4, 1.1])
    Ut = np.stack([O.split_tree(-1j * (Heff + E * Hd), 2.0 * ln, deep) for E, ln in zip((2.0, 0.0, -1.0), lens)])
    T = float(lens.sum())
    ens = O.Ensemble(Ut, L, [1.0], H + Hd, None, T, n, seed=21, record=2, rec_cap=20000, branch_len=lens)
    ens.init(0, 0)
    eng = q.Engine(Ut, L, [1.0], H + Hd, None, T, n, seed=21, record=2, rec_cap=64, max_dumps=1, branch_len=lens)
    eng.set_states(start_states(n, d))
    eng.init_thresholds()
    assert ens.run_periods(3) == 0
    eng.run_periods(3)
    psi, t, eta, jc = eng.states()
    assert jc.sum() > 10
    np.testing.assert_allclose(t, 3 * T, rtol=1e-12)
    assert np.array_equal(psi, ens.phi) and np.array_equal(t, ens.t) and np.array_equal(eta, ens.eta)
    for tr in range(n):
        for a, b in zip(eng.jumps(tr), ens.jumps(tr)):
            assert np.array_equal(a, b), tr
