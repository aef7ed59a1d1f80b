"""Batched engine (qjx_create_batch): ensembles of uneven dimension, parameters, seeds and sizes
advanced by the same micro-step launches.  Every trajectory, jump record and observable equals,
bit for bit, its run in an engine of its own and the oracle's."""
import numpy as np
import pytest

from oracle import oracle_py as O
from tests.helpers import T2PI, random_observable
from tests.test_gpu_parity import assert_same_observables

pytestmark = pytest.mark.gpu


def ensemble(N, E0, gamma, seed, n, deep, tr_base=0, A=1.5, U=0.5):
    H, Hd, L, K0, K1 = O.dimer_operators(N, 1.0, U, E0, A, gamma)
    Ut = np.stack([O.split_tree(K0, T2PI, deep), O.split_tree(K1, T2PI, deep)])
    d = N + 1
    return dict(U=Ut, L=L, g=[1.0], HE=H + E0 * Hd, R=np.stack([random_observable(d, seed)]), n_traj=n, T=T2PI,
                seed=seed, tr_base=tr_base)


def flow(eng, n, d_rows, starts, periods=3, dumps=(1, 3)):
    psi = np.zeros((n, d_rows), complex)
    psi[:, 0] = 1.0
    eng.set_states(psi)
    eng.init_thresholds()
    eng.run_periods(1, is_obs=0)
    eng.reset_times()
    eng.observe(0, is_start=True)
    eng.run_periods(periods, dump_at=list(dumps), dump_base=1)
    return eng.states(), [eng.observables(i, 1, want_adr=True) for i in range(1 + len(dumps))]


def test_batch_equals_alone_and_oracle():
    import os_d_b200 as q

    deep = 10
    specs = [(12, 0.3, 0.05, 3, 24, 0), (33, 1.7, 0.5, 4, 40, 100), (70, 1.0, 0.02, 5, 16, 7), (4, 0.0, 1.0, 6, 9, 0),
             (129, 0.6, 0.2, 8, 12, 3)]
    ens = [ensemble(N, E0, gm, sd, n, deep, tb) for N, E0, gm, sd, n, tb in specs]
    B = q.Engine.batch(ens, deep=deep, record=2, rec_cap=64, keep_adr=1, max_dumps=3)
    (psi_b, t_b, eta_b, jc_b), obs_b = flow(B, B.n, B.d, None)
    total_jumps = 0
    for e, x in enumerate(ens):
        r, d, n = B.ranges[e], x["U"].shape[-1], x["n_traj"]
        # alone
        A = q.Engine(x["U"], x["L"], x["g"], x["HE"], x["R"], x["T"], n, seed=x["seed"], tr_base=x["tr_base"],
                     record=2, rec_cap=64, keep_adr=1, max_dumps=3)
        (psi_a, t_a, eta_a, jc_a), obs_a = flow(A, n, d, None)
        assert np.array_equal(psi_b[r, :d], psi_a) and not np.any(psi_b[r, d:])
        assert np.array_equal(t_b[r], t_a) and np.array_equal(eta_b[r], eta_a) and np.array_equal(jc_b[r], jc_a)
        for i in range(n):
            for a, b in zip(B.jumps(r.start + i), A.jumps(i)):
                assert np.array_equal(a, b), (e, i)
        for ob, oa in zip(obs_b, obs_a):
            for k in ("norm", "mean", "dispersion", "m2", "energy"):
                assert np.array_equal(ob[k][0, r], oa[k][0]), (e, k)
            assert np.array_equal(ob["random_obs"][0, r], oa["random_obs"][0])
            assert np.array_equal(ob["adr"][0, r, :d], oa["adr"][0])
        # oracle
        o = O.Ensemble(x["U"], x["L"], x["g"], x["HE"], x["R"], x["T"], n, seed=x["seed"], record=2, rec_cap=20000,
                       tr_base=x["tr_base"])
        o.init(0, 0)
        assert o.run_periods(1, is_obs=0) == 0
        o.t[:] = 0.0
        res = [o.observables(is_start=True, want_adr=True)]
        assert o.run_periods(1) == 0
        res.append(o.observables(want_adr=True))
        assert o.run_periods(2) == 0
        res.append(o.observables(want_adr=True))
        assert np.array_equal(o.phi, psi_a) and np.array_equal(o.jumps_counts, jc_a)
        for oo, oa in zip(res, obs_a):
            assert_same_observables(oo, oa)
        total_jumps += int(jc_a.sum())
    assert total_jumps > 0


def test_batch_of_one_is_the_ordinary_engine():
    import os_d_b200 as q

    x = ensemble(20, 1.0, 0.1, 9, 32, 12, tr_base=5)
    B = q.Engine.batch([x], deep=12, record=1, keep_adr=1, max_dumps=3)
    A = q.Engine(x["U"], x["L"], x["g"], x["HE"], x["R"], x["T"], 32, seed=9, tr_base=5, record=1, keep_adr=1,
                 max_dumps=3)
    (sb, ob), (sa, oa) = flow(B, 32, 21, None), flow(A, 32, 21, None)
    for a, b in zip(sb, sa):
        assert np.array_equal(a, b)
    for x1, x2 in zip(ob, oa):
        for k in x1:
            assert np.array_equal(x1[k], x2[k]), k


def test_batched_lyapunov_sweep_equals_single_runs():
    """LpnMult over a batch of parameter points (the production sweep as one launch): every
    ensemble's states and Lyapunov values equal its own single-ensemble run, bit for bit."""
    import os_d_b200 as q
    from tests.test_lpn_cpu import CFGS

    cfg = dict(CFGS[1])
    deep = 10
    specs = [(20, 1.0, 0.1, 3, 10, 0), (33, 1.0, 0.3, 4, 14, 50), (12, 0.5, 0.05, 5, 8, 7)]
    ens = [ensemble(N, E0, gm, sd, n, deep, tb, U=0.3 + 0.1 * i) for i, (N, E0, gm, sd, n, tb) in enumerate(specs)]

    def flow(eng, rows):
        psi = np.zeros((eng.n, rows), complex)
        psi[:, 0] = 1.0
        eng.set_states(psi)
        eng.init_thresholds()
        eng.set_bases_only(True)
        eng.run_periods(1, is_obs=0)
        eng.set_bases_only(False)
        eng.lpn_start(**cfg)
        eng.reset_times()
        for p in range(3):
            eng.run_periods(1)
            eng.lpn_period((p + 1) * T2PI)
        return eng.states(), eng.lpn_values()

    B = q.Engine.batch(ens, deep=deep, record=1, max_dumps=1)
    (psi_b, t_b, eta_b, jc_b), lv_b = flow(B, B.d)
    renorms = 0
    for e, x in enumerate(ens):
        r, d = B.ranges[e], x["U"].shape[-1]
        A = q.Engine(x["U"], x["L"], x["g"], x["HE"], x["R"], x["T"], x["n_traj"], seed=x["seed"],
                     tr_base=x["tr_base"], record=1, max_dumps=1)
        (psi_a, t_a, eta_a, jc_a), lv_a = flow(A, d)
        assert np.array_equal(psi_b[r, :d], psi_a) and np.array_equal(t_b[r], t_a) and np.array_equal(eta_b[r], eta_a)
        for k in lv_a:
            assert np.array_equal(lv_b[k][r], lv_a[k]), (e, k)
        renorms += int(lv_a["num_renorms"].sum())
    assert renorms > 0


def test_split_batch_equals_split_alone():
    """Split precision in the batched engine: ensembles of uneven dimension (d 13 to 201) share the
    tcgen05 micro-steps, each with its own padded tiles and bf16 planes; every trajectory's state,
    jump record and observable equals, bit for bit, the same ensemble run alone in split precision
    (tiles never mix trajectories' arithmetic), FP64 rechecks included."""
    import os_d_b200 as q

    deep = 12
    specs = [(12, 0.3, 0.05, 3, 24, 0), (200, 1.0, 0.1, 4, 160, 100), (70, 1.0, 0.02, 5, 16, 7),
             (33, 1.7, 0.5, 6, 40, 0)]
    ens = [ensemble(N, E0, gm, sd, n, deep, tb) for N, E0, gm, sd, n, tb in specs]
    B = q.Engine.batch(ens, deep=deep, record=2, rec_cap=64, keep_adr=1, max_dumps=3, precision=1)
    (psi_b, t_b, eta_b, jc_b), obs_b = flow(B, B.n, B.d, None)
    st_b = B.stats()
    assert st_b["rechecks"] > 0 and jc_b.sum() > 0
    for e, x in enumerate(ens):
        r, d, n = B.ranges[e], x["U"].shape[-1], x["n_traj"]
        A = q.Engine(x["U"], x["L"], x["g"], x["HE"], x["R"], x["T"], n, seed=x["seed"], tr_base=x["tr_base"],
                     record=2, rec_cap=64, keep_adr=1, max_dumps=3, precision=1)
        (psi_a, t_a, eta_a, jc_a), obs_a = flow(A, n, d, None)
        assert np.array_equal(psi_b[r, :d], psi_a) and not np.any(psi_b[r, d:])
        assert np.array_equal(t_b[r], t_a) and np.array_equal(eta_b[r], eta_a) and np.array_equal(jc_b[r], jc_a)
        for i in range(n):
            for a, b in zip(B.jumps(r.start + i), A.jumps(i)):
                assert np.array_equal(a, b), (e, i)
        for ob, oa in zip(obs_b, obs_a):
            for k in ("norm", "mean", "dispersion", "m2", "energy"):
                assert np.array_equal(ob[k][0, r], oa[k][0]), (e, k)
            assert np.array_equal(ob["random_obs"][0, r], oa["random_obs"][0])
        A.close()
    B.close()
