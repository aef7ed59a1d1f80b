"""GPU engine versus the CPU oracle on identical inputs (bit-exact FP64 trajectories).

The engine and the oracle share one arithmetic contract (k-ascending fma chains in every
matvec, literal sequential norms), so with the same propagators and the same uniform
sequences every jump time, channel, norm, eta, final state and observable is bit-identical.
"""
import numpy as np
import pytest

from oracle import oracle_py as O
from tests.helpers import dimer_problem, random_observable, start_states

pytestmark = pytest.mark.gpu


def _engine_mod():
    import os_d_b200  # fails loudly when the native library is missing

    return os_d_b200


def run_pair(N, n, periods, seed=42, record=2, deep=16, nr=1, tp=0, dumps=(), start_type=0, rng_kind=0,
             inj=None, params=None):
    q = _engine_mod()
    P = dimer_problem(N, deep=deep, **(params or {}))
    d = P["d"]
    R = np.stack([random_observable(d, 7 + i) for i in range(nr)]) if nr else None
    inj_u, inj_off = inj if inj is not None else (None, None)
    ens = O.Ensemble(P["U"], P["L"], [1.0], P["HE"], R, P["T"], n, seed=seed, record=record, rng_kind=rng_kind,
                     inj_u=inj_u, inj_off=inj_off, rec_cap=20000)
    ens.init(start_type, 0)
    max_dumps = 1 + len(dumps)
    eng = q.Engine(P["U"], P["L"], [1.0], P["HE"], R, P["T"], n, seed=seed, record=record, rng_kind=rng_kind,
                   rec_cap=64, keep_adr=1, max_dumps=max_dumps)
    eng.set_states(start_states(n, d, start_type, 0))
    if rng_kind == 1:
        eng.set_uniforms(inj_u, inj_off)
    eng.init_thresholds()
    # transient without recording, then reset times, dump 0 with start semantics
    if tp:
        assert ens.run_periods(tp, is_obs=0) == 0
        eng.run_periods(tp, is_obs=0)
    ens.t[:] = 0.0
    eng.reset_times()
    ob0 = ens.observables(is_start=True, want_adr=True)
    eng.observe(0, is_start=True)
    results = [(ob0, eng.observables(0, 1, want_adr=True))]
    # observation periods with in-kernel dumps
    prev = 0
    o_dumps = []
    for p in dumps:
        assert ens.run_periods(p - prev, is_obs=1) == 0
        prev = p
        o_dumps.append(ens.observables(want_adr=True))
    assert ens.run_periods(periods - prev, is_obs=1) == 0
    eng.run_periods(periods, is_obs=1, dump_at=list(dumps), dump_base=1)
    for i, od in enumerate(o_dumps):
        results.append((od, eng.observables(1 + i, 1, want_adr=True)))
    return ens, eng, results


def assert_same_trajectories(ens, eng, record=2):
    psi, t, eta, jc = eng.states()
    assert np.array_equal(t, ens.t), np.abs(t - ens.t).max()
    assert np.array_equal(eta, ens.eta)
    assert np.array_equal(psi, ens.phi), np.abs(psi - ens.phi).max()
    if record:
        assert np.array_equal(jc, ens.jumps_counts)
        for tr in range(ens.n):
            t_o, ty_o, n_o, e_o = ens.jumps(tr)
            t_g, ty_g, n_g, e_g = eng.jumps(tr)
            assert np.array_equal(t_g, t_o), tr
            assert np.array_equal(ty_g, ty_o), tr
            assert np.array_equal(n_g, n_o), tr
            assert np.array_equal(e_g, e_o), tr


def assert_same_observables(o, g):
    for k in ("norm", "mean", "dispersion", "m2", "energy"):
        assert np.array_equal(g[k][0], o[k]), (k, np.abs(g[k][0] - o[k]).max())
    assert np.array_equal(g["random_obs"][0], o["random_obs"])
    assert np.array_equal(g["adr"][0], o["adr"])


def test_small_dimer_bit_exact():
    ens, eng, res = run_pair(N=20, n=64, periods=4)
    assert_same_trajectories(ens, eng)
    assert ens.jumps_counts.sum() > 0
    for o, g in res:
        assert_same_observables(o, g)


def test_transient_and_dumps_bit_exact():
    ens, eng, res = run_pair(N=30, n=50, periods=6, tp=2, dumps=(1, 3, 6))
    assert_same_trajectories(ens, eng)
    assert len(res) == 4
    for o, g in res:
        assert_same_observables(o, g)


def test_config1_dim101_bit_exact():
    # dimer N=100 (dim 101) of the CPU-runnable configuration, sampled to 96 trajectories x 3 periods
    ens, eng, res = run_pair(N=100, n=96, periods=3, seed=42)
    assert_same_trajectories(ens, eng)
    for o, g in res:
        assert_same_observables(o, g)


def test_dim201_bit_exact():
    ens, eng, res = run_pair(N=200, n=40, periods=1, seed=7, nr=0)
    assert_same_trajectories(ens, eng)


def test_injected_uniforms_bit_exact():
    n, N = 33, 16
    rng = np.random.default_rng(3)
    lens = rng.integers(400, 600, size=n)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    u = rng.random(off[-1])
    u[u == 0.0] = 0.5
    ens, eng, res = run_pair(N=N, n=n, periods=2, rng_kind=1, inj=(u, off), nr=0)
    assert_same_trajectories(ens, eng)


def test_uniform_start_state_and_record_off():
    ens, eng, res = run_pair(N=24, n=40, periods=3, record=0, start_type=1, nr=2)
    assert_same_trajectories(ens, eng, record=0)
    for o, g in res:
        assert_same_observables(o, g)


def test_record_buffer_overflow_drains_and_resumes():
    # rec_cap 64 on the device with >64 jumps per trajectory forces pause / drain / resume
    ens, eng, _ = run_pair(N=60, n=20, periods=3, nr=0)
    assert ens.jumps_counts.max() > 64
    assert_same_trajectories(ens, eng)


def test_rng_exhaustion_reports_error():
    q = _engine_mod()
    P = dimer_problem(12)
    n = 4
    off = np.array([0, 5, 10, 15, 20], np.int64)
    u = np.full(20, 0.5)
    eng = q.Engine(P["U"], P["L"], [1.0], P["HE"], None, P["T"], n, rng_kind=1, record=1)
    eng.set_states(start_states(n, P["d"]))
    eng.set_uniforms(u, off)
    eng.init_thresholds()
    with pytest.raises(q.QjxError, match="exhausted"):
        eng.run_periods(50, is_obs=1)
