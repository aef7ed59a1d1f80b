"""Lyapunov paired trajectories (task_id 7, LpnMult) in the CPU oracle.

The oracle's orc_lpn_start / orc_lpn_period are checked against a numpy restatement written
directly from the reference's functions (var_trajectory_lpn, experiment.cpp:2278-2397;
lambda_lpn / lambda_lpn_now, experiment.cpp:3065-3135; calc_chars_lpn, core.cpp:764-785;
calc_delta_s / calc_delta_f, core.cpp:839-901), one call at a time from the same inputs, and
the oracle's exp10 / log against numpy's.
"""
import numpy as np
import pytest

from oracle import oracle_py as O
from tests.helpers import T2PI, dimer_problem, random_observable, start_states


def test_exp10_log_within_two_ulp():
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(-20, 20, 4000), np.linspace(-10, 10, 401), rng.uniform(-300, 300, 1000)])
    for x in xs:
        a, b = O.lpn_exp10(x), 10.0 ** x
        assert abs(a - b) <= 2 * np.spacing(b), x
    ys = np.concatenate([10 ** rng.uniform(-300, 300, 4000), rng.uniform(0.5, 2, 4000), [5e-324, 1e-310, 1.0]])
    for y in ys:
        a, b = O.lpn_log(y), np.log(y)
        assert abs(a - b) <= 2 * np.spacing(abs(b)) if b != 0 else a == 0.0, y
    assert O.lpn_log(0.0) == -np.inf and O.lpn_log(np.inf) == np.inf and np.isnan(O.lpn_log(-1.0))
    assert O.lpn_exp10(0.0) == 1.0 and O.lpn_exp10(-400.0) == 0.0


# ------------------------------------------------------------------ numpy restatement
def chars(phi, HE, R):
    nrm = np.sum(phi.real ** 2 + phi.imag ** 2)
    adr = (phi.real ** 2 + phi.imag ** 2) / nrm
    xh = phi / np.sqrt(nrm)
    y = HE @ xh
    energy = np.sum(xh.real * y.real + xh.imag * y.imag)
    robs = np.array([np.vdot(xh, Ro @ xh) for Ro in R])
    return dict(mean=np.sum(np.arange(len(phi)) * adr), energy=energy, robs=robs)


def delta(cfg, cv, cb, d):
    t = cfg["lpn_type"]
    if t == -1:
        return abs(cv["mean"] - cb["mean"]) / d
    if t == -2:
        return abs(cv["energy"] - cb["energy"]) / cfg["max_energy"]
    return abs(cb["robs"][t] - cv["robs"][t])


def var_trajectory(cfg, base, phi_v, v, var_pos, HE, R):
    d = len(base)
    u = np.array([O.philox_uniform(777, (1 << 63) | v, var_pos + i) for i in range(2 * d)])
    w = (2 * u[:d] - 1) + 1j * (2 * u[d:] - 1)
    w = w / np.sqrt(np.sum(np.abs(w) ** 2))
    n2 = np.sum(np.abs(base) ** 2)
    lo, hi = cfg["eps_low"], cfg["eps_high"]
    diff, deep = hi - lo, 0
    eps = 10.0 ** ((lo + hi) * 0.5)
    cb = chars(base, HE, R)
    phi = phi_v.copy()
    while deep < cfg["eps_deep"]:
        phi = base + eps * w
        phi = phi / np.sqrt(np.sum(np.abs(phi) ** 2)) * np.sqrt(n2)
        ds = delta(cfg, chars(phi, HE, R), cb, d)
        if abs(ds - cfg["delta_s"]) < cfg["eps_error"]:
            break
        if ds > cfg["delta_s"]:
            hi -= 0.5 * diff
        elif ds < cfg["delta_s"]:
            lo += 0.5 * diff
        else:
            break
        diff = hi - lo
        deep += 1
        eps = 10.0 ** ((lo + hi) * 0.5)
    return phi, var_pos + 2 * d, deep


def lambda_step(cfg, phi_b, phi_v, v, var_pos, lam, ds, curr_time, HE, R):
    """lambda_lpn (per_period 0) / lambda_lpn_now (1) of one variation."""
    d = len(phi_b)
    cb = chars(phi_b, HE, R)
    df = delta(cfg, chars(phi_v, HE, R), cb, d)
    if cfg["per_period"] or df > max(cfg["delta_f_high"], ds * 10.0) or df < cfg["delta_f_low"]:
        lam = lam + np.log(df / ds + 1e-16)
        phi_v, var_pos, _ = var_trajectory(cfg, phi_b, phi_v, v, var_pos, HE, R)
        ds_new = delta(cfg, chars(phi_v, HE, R), cb, d)
        return dict(phi=phi_v, var_pos=var_pos, lam=lam, ds=ds_new, now=lam / curr_time, renorm=1, df=df)
    return dict(phi=phi_v, var_pos=var_pos, lam=lam, ds=ds, now=(lam + np.log(df / ds + 1e-16)) / curr_time,
                renorm=0, df=df)


CFGS = [
    dict(lpn_type=-1, eps_deep=60, per_period=0, eps_low=-10.0, eps_high=10.0, eps_error=1e-10, delta_s=1e-3,
         delta_f_high=5e-3, delta_f_low=5e-4, max_energy=1.0),
    dict(lpn_type=0, eps_deep=100, per_period=0, eps_low=-10.0, eps_high=10.0, eps_error=1e-10, delta_s=1e-3,
         delta_f_high=1e-1, delta_f_low=8e-4, max_energy=1.0),
    dict(lpn_type=-2, eps_deep=30, per_period=1, eps_low=-8.0, eps_high=2.0, eps_error=1e-12, delta_s=1e-4,
         delta_f_high=1e-1, delta_f_low=1e-5, max_energy=None),
]


@pytest.mark.parametrize("cfg", CFGS, ids=["mean", "robs", "energy-per-period"])
def test_oracle_lpn_matches_numpy_restatement(cfg):
    cfg = dict(cfg)
    N, n, tp, periods = 12, 8, 2, 6
    P = dimer_problem(N, deep=10)
    d, half = P["d"], n // 2
    if cfg["max_energy"] is None:
        cfg["max_energy"] = float(np.max(np.abs(np.diag(P["H"]).real)))
    R = np.stack([random_observable(d, 5)])
    ens = O.Ensemble(P["U"], P["L"], [1.0], P["HE"], R, P["T"], n, seed=3, record=0)
    ens.init(0, 0)
    assert ens.run_periods(tp, is_obs=0, tr0=0, tr1=half) == 0
    ens.t[:] = 0.0
    lp = O.Lpn(ens, **cfg)
    before = ens.phi.copy()
    lp.start()
    # start: every variation is its base's copy perturbed to delta_s, with the base's jump stream
    assert np.array_equal(ens.rng_src[half:], np.arange(half, dtype=np.int32))
    assert np.array_equal(ens.rng_pos[half:], ens.rng_pos[:half]) and np.array_equal(ens.eta[half:], ens.eta[:half])
    assert np.array_equal(ens.phi[:half], before[:half])
    for b in range(half):
        v = half + b
        phi, pos, deep = var_trajectory(cfg, before[b], before[b], v, 0, P["HE"], R)
        assert pos == lp.var_pos[v] and deep == lp.eps_iters[v]
        np.testing.assert_allclose(ens.phi[v], phi, rtol=0, atol=1e-13)
        np.testing.assert_allclose(np.sum(np.abs(ens.phi[v]) ** 2), np.sum(np.abs(before[b]) ** 2), rtol=1e-13)
        cb, cv = chars(before[b], P["HE"], R), chars(phi, P["HE"], R)
        np.testing.assert_allclose(lp.a["delta_s"][v], delta(cfg, cv, cb, d), rtol=1e-9)
        if deep < cfg["eps_deep"]:
            assert abs(lp.a["delta_s"][v] - cfg["delta_s"]) < cfg["eps_error"] * 1.01
        np.testing.assert_allclose(lp.a["mean_lpn"][v], cv["mean"], rtol=1e-12)
    renorms = 0
    for p in range(periods):
        assert ens.run_periods(1, is_obs=1) == 0
        phi0, pos0 = ens.phi.copy(), lp.var_pos.copy()
        lam0, ds0 = lp.a["lambda"].copy(), lp.a["delta_s"].copy()
        curr_time = (p + 1) * P["T"]
        lp.period(curr_time)
        for b in range(half):
            v = half + b
            r = lambda_step(cfg, phi0[b], phi0[v], v, pos0[v], lam0[v], ds0[v], curr_time, P["HE"], R)
            assert r["renorm"] == lp.renormed[v], (p, v)
            renorms += r["renorm"]
            assert r["var_pos"] == lp.var_pos[v]
            np.testing.assert_allclose(ens.phi[v], r["phi"], rtol=0, atol=1e-12)
            np.testing.assert_allclose(lp.a["lambda"][v], r["lam"], rtol=1e-10, atol=1e-12)
            np.testing.assert_allclose(lp.a["lambda_now"][v], r["now"], rtol=1e-9, atol=1e-12)
            np.testing.assert_allclose(lp.a["delta_s"][v], r["ds"], rtol=1e-8)
            if r["renorm"]:
                assert ens.rng_pos[v] == ens.rng_pos[b] and ens.eta[v] == ens.eta[b]
                np.testing.assert_allclose(lp.a["df_rec"][v], r["df"], rtol=1e-9)
    assert lp.num_renorms[half:].sum() == renorms and renorms > 0
    if cfg["per_period"]:
        assert renorms == half * periods
    assert np.all(lp.num_renorms[:half] == 0) and np.all(lp.a["lambda_now"][:half] == 0)


def test_variation_replays_base_stream_without_perturbation():
    """eps = 10^-400 = 0 and no bisection: the variation is the base (rescaled by |base| / |base|)
    and, drawing the base's jump stream, it makes the same jumps at the same times."""
    N, n = 8, 4
    P = dimer_problem(N, deep=10)
    ens = O.Ensemble(P["U"], P["L"], [1.0], P["HE"], None, P["T"], n, seed=11, record=1)
    ens.init(0, 0)
    assert ens.run_periods(1, is_obs=0, tr0=0, tr1=2) == 0
    ens.t[:] = 0.0  # resresh_times
    lp = O.Lpn(ens, lpn_type=-1, eps_deep=1, eps_low=-400.0, eps_high=-400.0, eps_error=1.0)
    lp.start()
    np.testing.assert_allclose(ens.phi[2:], ens.phi[:2], rtol=0, atol=1e-15)
    assert ens.run_periods(3, is_obs=1) == 0
    for b in range(2):
        tb, kb, _, _ = ens.jumps(b)
        tv, kv, _, _ = ens.jumps(2 + b)
        assert len(tb) > 0 and np.array_equal(kb, kv)
        np.testing.assert_allclose(tv, tb, rtol=0, atol=1e-9)
