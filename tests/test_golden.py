"""Golden fixture (tests/golden/qj_dim11_seed42.npz, made by tests/golden/make_golden.py):
the oracle and the GPU engine must reproduce it bit for bit."""
import os

import numpy as np
import pytest

from tests.golden.make_golden import N, compute, deep, n, periods, seed, tp

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "qj_dim11_seed42.npz")


def test_oracle_reproduces_golden_fixture():
    g = np.load(GOLD)
    out = compute()
    for k in g.files:
        assert np.array_equal(out[k], g[k]), k


@pytest.mark.gpu
def test_engine_reproduces_golden_fixture():
    import os_d_b200 as q

    g = np.load(GOLD)
    H, Hd, L, Ut = q.build_dimer(N, 1.0, 0.5, 1.0, 1.5, 0.1, 1.0, deep)
    T = 2.0 * 3.1415926535897932384626433832795
    eng = q.Engine(Ut, L, [1.0], H + Hd, None, T, n, seed=seed, record=2, max_dumps=periods + 1)
    psi0 = np.zeros((n, N + 1), np.complex128)
    psi0[:, 0] = 1
    eng.set_states(psi0)
    eng.init_thresholds()
    eng.run_periods(tp, is_obs=0)
    eng.reset_times()
    eng.observe(0, is_start=True)
    eng.run_periods(periods, is_obs=1, dump_at=list(range(1, periods + 1)), dump_base=1)
    psi, t, eta, jc = eng.states()
    assert np.array_equal(psi, g["psi"]) and np.array_equal(t, g["t"]) and np.array_equal(eta, g["eta"])
    assert np.array_equal(jc, g["jumps_counts"])
    ob = eng.observables(0, periods + 1)
    for k in ("norm", "mean", "dispersion", "m2", "energy"):
        assert np.array_equal(ob[k], g["obs_" + k]), k
    jt = np.concatenate([eng.jumps(tr)[0] for tr in range(n)])
    assert np.array_equal(jt, g["jump_times"])
    assert np.array_equal(np.concatenate([eng.jumps(tr)[1] for tr in range(n)]), g["diss_types"])
