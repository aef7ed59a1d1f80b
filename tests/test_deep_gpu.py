"""Deep tasks (task_id 4, StdDeep): every half period runs as 2 deep_num_steps units of the split
tree of T / (2 deep_num_steps) and the observables are taken after every sub-period
(ex_period_obs_deep, source/cpp/QJX/QJX/core.cpp:114-153).  GPU against the oracle on the same
inputs, bit for bit."""
import numpy as np
import pytest

from oracle import oracle_py as O
from tests.helpers import T2PI, start_states

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,nsub,periods,tp", [(14, 2, 2, 1), (40, 3, 1, 0)])
def test_deep_task_bit_exact(N, nsub, periods, tp):
    import os_d_b200 as q

    n, deep, seed = 40, 16, 9
    H, Hd, L, K0, K1 = O.dimer_operators(N, 1.0, 0.5, 1.0, 1.5, 0.1)
    t_head = 0.5 * T2PI / nsub
    Ut = np.stack([O.split_tree(K0, t_head, deep), O.split_tree(K1, t_head, deep)])
    HE = H + 1.0 * Hd
    d = N + 1
    ens = O.Ensemble(Ut, L, [1.0], HE, None, t_head, n, seed=seed, record=2, rec_cap=20000)
    ens.init(0, 0)
    ndump = periods * 2 * nsub
    eng = q.Engine(Ut, L, [1.0], HE, None, T2PI, n, seed=seed, record=2, rec_cap=64, keep_adr=1,
                   max_dumps=1 + ndump, deep_num_steps=nsub)
    eng.set_states(start_states(n, d))
    eng.init_thresholds()
    for _ in range(tp):  # transient: whole periods, no observables
        for b in range(2):
            assert ens.run_branch_units(b, 2 * nsub, is_obs=0) == 0
        eng.run_periods(1, is_obs=0)
    ens.t[:] = 0.0
    eng.reset_times()
    eng.observe(0, is_start=True)
    obs = [ens.observables(is_start=True, want_adr=True)]
    for _ in range(periods):
        for b in range(2):
            for _ in range(nsub):
                assert ens.run_branch_units(b, 2) == 0
                obs.append(ens.observables(want_adr=True))
    eng.run_periods(periods, dump_base=1)
    psi, t, eta, jc = eng.states()
    assert jc.sum() > 0
    assert np.array_equal(psi, ens.phi) and np.array_equal(t, ens.t) and np.array_equal(jc, ens.jumps_counts)
    for tr in range(n):
        for a, b in zip(eng.jumps(tr), ens.jumps(tr)):
            assert np.array_equal(a, b), tr
    assert len(obs) == 1 + ndump
    for i, o in enumerate(obs):
        g = eng.observables(i, 1, want_adr=True)
        for k in ("norm", "mean", "dispersion", "m2", "energy"):
            assert np.array_equal(g[k][0], o[k]), (i, k)
        assert np.array_equal(g["adr"][0], o["adr"]), i
