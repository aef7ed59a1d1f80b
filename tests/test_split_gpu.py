"""Split-precision form (precision 1: bf16x3 tcgen05 matvecs, FP64 norms and state) against the
complex FP64 plain form on the same inputs.  The split form is not bit-exact: its tolerances are
stated per test.  Trajectories whose norm crosses its threshold in a different bisection bin
diverge, so trajectory-level comparisons use the trajectories whose jump counts agree."""
import numpy as np
import pytest

from tests.helpers import dimer_problem, start_states

pytestmark = pytest.mark.gpu


def run(P, n, periods, precision, seed=3, split_recheck=0.0, want_stats=False):
    import os_d_b200 as q

    eng = q.Engine(P["U"], P["L"], [1.0], P["HE"], None, P["T"], n, seed=seed, record=1, max_dumps=2, rec_cap=4096,
                   keep_adr=1, precision=precision, split_recheck=split_recheck)
    eng.set_states(start_states(n, P["d"], 0, 0))
    eng.init_thresholds()
    eng.observe(0, is_start=True)
    eng.run_periods(periods, dump_at=[periods], dump_base=1)
    psi, t, eta, jc = eng.states()
    obs = eng.observables(1, 1)
    st = eng.stats()
    eng.close()
    return (psi, jc, obs, st) if want_stats else (psi, jc, obs)


@pytest.mark.parametrize("N", [20, 200])
def test_split_recheck_of_every_step_reproduces_fp64_bit_for_bit(N):
    """With dissipation too weak for a jump in 2 periods (g = 1e-7: the norm decays by about 1e-4,
    far above the rounding of a unitary step, which would carry an FP64 norm above 1 and make the
    plain form reject it as the reference does) every norm test passes, and a recheck band of 1
    sends every step to the FP64 recheck, whose product follows the plain form's arithmetic: the
    states after 2 periods equal the plain form's bit for bit, and every matvec of the run was
    taken twice."""
    P = dimer_problem(N, g=1e-7)
    psi_s, jc_s, _, st = run(P, 40, 2, 1, split_recheck=1.0, want_stats=True)
    psi_d, jc_d, _ = run(P, 40, 2, 0)
    assert jc_s.sum() == 0 and jc_d.sum() == 0
    assert np.array_equal(psi_s, psi_d)
    assert st["rechecks"] == 40 * 2 * 4  # 2 periods x 2 branches x 2 level-0 steps


def test_split_without_recheck_runs_and_counts_none():
    P = dimer_problem(20)
    psi, jc, _, st = run(P, 64, 2, 1, split_recheck=-1.0, want_stats=True)
    assert st["rechecks"] == 0 and jc.sum() > 0
    nrm = np.linalg.norm(psi, axis=1)
    assert np.all(np.isfinite(nrm)) and nrm.max() < 1 + 1e-4 and nrm.min() > 0


def test_split_unitary_dynamics_matches_fp64():
    # g = 0: no dissipation, no jumps; 2 periods = 8 matvecs per trajectory
    P = dimer_problem(20, g=0.0)
    psi_s, jc_s, _ = run(P, 64, 2, 1)
    psi_d, jc_d, _ = run(P, 64, 2, 0)
    assert jc_s.sum() == 0 and jc_d.sum() == 0
    assert np.abs(psi_s - psi_d).max() < 1e-4  # bf16x3 with FP32 accumulation: ~1e-6 per matvec
    assert np.abs(np.linalg.norm(psi_s, axis=1) - 1).max() < 1e-4


@pytest.mark.parametrize("N,n,periods", [(20, 256, 2), (200, 512, 1)])
def test_split_dissipative_ensemble_close_to_fp64(N, n, periods):
    P = dimer_problem(N)
    psi_s, jc_s, o_s = run(P, n, periods, 1)
    psi_d, jc_d, o_d = run(P, n, periods, 0)
    assert jc_d.sum() > 0
    same = jc_s == jc_d
    assert same.mean() > 0.8, same.mean()
    # trajectories with the same jump sequence stay close to the FP64 ones
    dev = np.abs(psi_s[same] - psi_d[same]).max(axis=1)
    assert np.median(dev) < 1e-3, np.median(dev)
    # the ensemble mean of <n1 - n2> agrees within the split-form tolerance of this short run
    m_s, m_d = o_s["mean"][0].mean(), o_d["mean"][0].mean()
    assert abs(m_s - m_d) < 0.02 * N, (m_s, m_d)


def test_autotuner_picks_and_caches_a_fitting_shape(tmp_path, monkeypatch):
    """qjx_autotune times every fitting tile shape of the split and plain forms at d = 41 and
    stores the fastest under (precision, d); a later engine with default tiles picks it from the
    cache, and its results equal an engine with the rule's shapes (tiles never change results)."""
    import os_d_b200 as q

    monkeypatch.setenv("QJX_TILE_CACHE", str(tmp_path / "tiles.txt"))
    P = dimer_problem(40)
    for precision in (0, 1):
        best, table = q.autotune(P["U"], P["L"], [1.0], P["HE"], T=P["T"], n_traj=512, precision=precision,
                                 n_periods=1)
        assert len(table) >= 4 and all(us > 0 for _, us in table)
        assert min(table, key=lambda x: x[1])[0] == best
    lines = (tmp_path / "tiles.txt").read_text().split("\n")
    assert lines[0].startswith("0 41 ") and lines[1].startswith("1 41 ")
    for precision in (0, 1):
        psi_c, jc_c, _ = run(P, 256, 2, precision)  # default tiles: the cached choice
        monkeypatch.setenv("QJX_TILE_CACHE", str(tmp_path / "none.txt"))
        psi_r, jc_r, _ = run(P, 256, 2, precision)  # the rule
        monkeypatch.setenv("QJX_TILE_CACHE", str(tmp_path / "tiles.txt"))
        assert np.array_equal(psi_c, psi_r) and np.array_equal(jc_c, jc_r)


def test_split_per_step_launches_equal_the_multi_step_launch(monkeypatch):
    """The split form runs a batch of micro-steps as one cooperative launch with grid barriers
    between them; when that launch cannot make every CTA resident it falls back to one launch per
    micro-step (forced here with QJX_SPLIT_COOP=0). Both give the same trajectories, jump records
    and observables, bit for bit, with jumps and FP64 rechecks in the run."""
    P = dimer_problem(40, g=0.3)
    a = run(P, 300, 3, 1, want_stats=True)
    monkeypatch.setenv("QJX_SPLIT_COOP", "0")
    b = run(P, 300, 3, 1, want_stats=True)
    assert a[1].sum() > 0 and a[3]["rechecks"] > 0
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    for k in ("norm", "mean", "energy"):
        assert np.array_equal(a[2][k], b[2][k]), k
    assert a[3]["micro_steps"] == b[3]["micro_steps"]
    assert b[3]["launches"] > a[3]["launches"]
