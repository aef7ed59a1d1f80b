"""Dimensions above 208 (N up to 1023): the plain step kernel narrows its sub-tiles (32, 16 or 8
trajectory columns) and propagator slabs to fit shared memory; trajectories, jump records and
observables stay bit-identical to the oracle."""
import numpy as np
import pytest

from oracle import oracle_py as O
from tests.helpers import T2PI, random_observable
from tests.test_gpu_parity import assert_same_observables, assert_same_trajectories
from tests.test_lpn_cpu import CFGS

pytestmark = pytest.mark.gpu


def fast_problem(N, deep, J=1.0, U=0.5, E=1.0, A=1.5, g=0.1):
    """The dimer's split tree from scipy's expm (LAPACK-fast at d ~ 1000); the engine and the
    oracle receive the same matrices, so parity does not depend on how they were made."""
    import scipy.linalg

    H, Hd, L, K0, K1 = O.dimer_operators(N, J, U, E, A, g)
    dts, dt = [], 0.5 * T2PI
    for _ in range(deep):
        dt *= 0.5
        dts.append(dt)
    Ut = np.stack([np.stack([scipy.linalg.expm(K * x) for x in dts]) for K in (K0, K1)])
    return dict(H=H, Hd=Hd, L=L, U=Ut, HE=H + E * Hd, T=T2PI, d=N + 1)


@pytest.mark.parametrize("N,n,deep", [(256, 40, 16), (400, 24, 14), (1000, 8, 12)])
def test_large_dims_bit_exact(N, n, deep):
    import os_d_b200 as q

    P = fast_problem(N, deep)
    d = P["d"]
    R = np.stack([random_observable(d, 7)])
    ens = O.Ensemble(P["U"], P["L"], [1.0], P["HE"], R, P["T"], n, seed=5, record=2, rec_cap=20000)
    ens.init(0, 0)
    eng = q.Engine(P["U"], P["L"], [1.0], P["HE"], R, P["T"], n, seed=5, record=2, rec_cap=64, keep_adr=1,
                   max_dumps=2)
    psi = np.zeros((n, d), complex)
    psi[:, 0] = 1.0
    eng.set_states(psi)
    eng.init_thresholds()
    eng.reset_times()
    ens.t[:] = 0.0
    eng.observe(0, is_start=True)
    res = [(ens.observables(is_start=True, want_adr=True), eng.observables(0, 1, want_adr=True))]
    assert ens.run_periods(1, is_obs=1) == 0
    eng.run_periods(1, is_obs=1, dump_at=[1], dump_base=1)
    res.append((ens.observables(want_adr=True), eng.observables(1, 1, want_adr=True)))
    assert_same_trajectories(ens, eng)
    assert ens.jumps_counts.sum() > 0
    for o, g in res:
        assert_same_observables(o, g)


def test_large_dim_rk_bit_exact():
    import os_d_b200 as q

    N, n, rk_ns = 230, 8, 5000
    H, Hd, L, K0, K1 = O.dimer_operators(N, 1.0, 0.5, 1.0, 1.5, 0.1)
    Heff = O.dimer_heff(N, 1.0, 0.5, 1.0, 0.1)
    d, T = N + 1, T2PI
    HE = H + Hd
    ens = O.Ensemble(np.zeros((2, 1, d, d)), L, [1.0], HE, None, T, n, seed=3, record=2, rec_cap=2000)
    ens.init(0, 0)
    assert ens.run_periods_rk(1, Heff, Hd, 1.0, 1.5, rk_ns) == 0
    eng = q.Engine.rk(Heff, Hd, L, [1.0], HE, None, T=T, n_traj=n, E0=1.0, A=1.5, rk_ns=rk_ns, seed=3, record=2)
    psi = np.zeros((n, d), complex)
    psi[:, 0] = 1.0
    eng.set_states(psi)
    eng.init_thresholds()
    eng.run_periods(1)
    assert_same_trajectories(ens, eng)


def test_large_dim_lpn_bit_exact():
    import os_d_b200 as q

    cfg = dict(CFGS[1])
    N, n = 500, 8
    P = fast_problem(N, 12)
    d, half, T = P["d"], n // 2, P["T"]
    R = np.stack([random_observable(d, 5)])
    ens = O.Ensemble(P["U"], P["L"], [1.0], P["HE"], R, T, n, seed=2, record=1, rec_cap=2000)
    ens.init(0, 0)
    assert ens.run_periods(1, is_obs=0, tr0=0, tr1=half) == 0
    lp = O.Lpn(ens, **cfg)
    lp.start()
    ens.t[:] = 0.0
    eng = q.Engine(P["U"], P["L"], [1.0], P["HE"], R, T, n, seed=2, record=1, max_dumps=2)
    psi = np.zeros((n, d), complex)
    psi[:, 0] = 1.0
    eng.set_states(psi)
    eng.init_thresholds()
    eng.set_active(half)
    eng.run_periods(1, is_obs=0)
    eng.set_active(n)
    eng.lpn_start(**cfg)
    eng.reset_times()
    for p in range(2):
        assert ens.run_periods(1, is_obs=1) == 0
        lp.period((p + 1) * T)
        eng.run_periods(1, is_obs=1)
        eng.lpn_period((p + 1) * T)
    psi_g, t, eta, _ = eng.states()
    assert np.array_equal(psi_g, ens.phi) and np.array_equal(t, ens.t) and np.array_equal(eta, ens.eta)
    g, o = eng.lpn_values(), lp.values()
    for k in ("lambda_now", "delta_s", "mean_lpn", "energy_lpn", "robs_lpn", "num_renorms"):
        assert np.array_equal(g[k], o[k]), k
