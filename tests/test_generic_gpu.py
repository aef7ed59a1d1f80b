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
