"""Lyapunov paired trajectories (task_id 7, LpnMult) on the GPU against the oracle, bit for bit:
the bases' transient alone (qjx_set_active), the start (copy + perturbation bisection), then every
observation period's lambda_lpn / lambda_lpn_now with renormalisations, the variations drawing
their bases' jump streams, and the observables of every dump."""
import numpy as np
import pytest

from oracle import oracle_py as O
from tests.helpers import dimer_problem, random_observable, start_states
from tests.test_lpn_cpu import CFGS

pytestmark = pytest.mark.gpu


def _equal_lpn(eng, lp, half):
    g, o = eng.lpn_values(), lp.values()
    for k in ("lambda_now", "lambda", "delta_s", "mean_lpn", "energy_lpn", "robs_lpn", "num_renorms"):
        assert np.array_equal(g[k], o[k]), k
    gl, ol = eng.lpn_last(), lp.last()
    for k in ("renormed", "ratio", "delta_s", "delta_f", "eps_iters", "eps"):
        assert np.array_equal(gl[k][half:], ol[k][half:]), k


@pytest.mark.parametrize("cfg", CFGS, ids=["mean", "robs", "energy-per-period"])
@pytest.mark.parametrize("N,n", [(20, 64), (60, 16)])
def test_lpn_bit_exact(cfg, N, n):
    import os_d_b200 as q

    cfg = dict(cfg)
    tp, periods, seed = 2, 5, 21
    P = dimer_problem(N, deep=12)
    d, half, T = P["d"], n // 2, P["T"]
    if cfg["max_energy"] is None:
        cfg["max_energy"] = float(np.max(np.abs(np.diag(P["H"]).real)))
    R = np.stack([random_observable(d, 5), random_observable(d, 6)])

    ens = O.Ensemble(P["U"], P["L"], [1.0], P["HE"], R, T, n, seed=seed, record=1, rec_cap=20000)
    ens.init(0, 0)
    assert ens.run_periods(tp, is_obs=0, tr0=0, tr1=half) == 0
    lp = O.Lpn(ens, **cfg)
    lp.start()
    ens.t[:] = 0.0
    obs = [ens.observables(is_start=True, want_adr=True)]

    eng = q.Engine(P["U"], P["L"], [1.0], P["HE"], R, T, n, seed=seed, record=1, keep_adr=1,
                   max_dumps=periods + 1)
    eng.set_states(start_states(n, d))
    eng.init_thresholds()
    eng.set_active(half)
    eng.run_periods(tp, is_obs=0)
    eng.set_active(n)
    eng.lpn_start(**cfg)
    eng.reset_times()
    eng.observe(0, is_start=True)
    psi, t, eta, _ = eng.states()
    assert np.array_equal(psi, ens.phi) and np.array_equal(eta, ens.eta)
    _equal_lpn(eng, lp, half)

    renorms = 0
    for p in range(periods):
        assert ens.run_periods(1, is_obs=1) == 0
        o = ens.observables(want_adr=True)  # calc_chars_std at the period end
        lp.period((p + 1) * T)
        after = ens.observables(want_adr=True)  # abs_diag_rho_all after lambda_lpn
        o["adr"][half:] = after["adr"][half:]
        obs.append(o)
        eng.run_periods(1, is_obs=1, dump_at=[1], dump_base=p + 1)
        eng.lpn_period((p + 1) * T, adr_dump=p + 1)
        psi, t, eta, jc = eng.states()
        assert np.array_equal(psi, ens.phi), p
        assert np.array_equal(t, ens.t) and np.array_equal(eta, ens.eta) and np.array_equal(jc, ens.jumps_counts)
        _equal_lpn(eng, lp, half)
        renorms += int(lp.renormed[half:].sum())
    assert renorms > 0
    for i, o in enumerate(obs):
        g = eng.observables(i, 1, want_adr=True)
        for k in ("norm", "mean", "dispersion", "m2", "energy"):
            assert np.array_equal(g[k][0], o[k]), (i, k)
        assert np.array_equal(g["random_obs"][0], o["random_obs"]), i
        assert np.array_equal(g["adr"][0], o["adr"]), i
    for tr in range(n):
        for a, b in zip(eng.jumps(tr), ens.jumps(tr)):
            assert np.array_equal(a, b), tr
