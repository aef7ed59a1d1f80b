"""Checkpoint / resume: a run interrupted after some periods, saved, loaded into a fresh engine
and continued equals the uninterrupted run bit for bit (states, times, thresholds, RNG cursors,
jump records after the restart, observables; Lyapunov pairs too)."""
import numpy as np
import pytest

from tests.helpers import dimer_problem, random_observable, start_states
from tests.test_lpn_cpu import CFGS

pytestmark = pytest.mark.gpu


def make(q, P, R, n, seed):
    e = q.Engine(P["U"], P["L"], [1.0], P["HE"], R, P["T"], n, seed=seed, record=2, keep_adr=1, max_dumps=2)
    e.set_states(start_states(n, P["d"]))
    e.init_thresholds()
    return e


def test_checkpoint_resume_is_bit_exact():
    import os_d_b200 as q

    P = dimer_problem(24, deep=12)
    R = random_observable(P["d"], 3)[None]
    n = 48
    full = make(q, P, R, n, 5)
    full.run_periods(3, is_obs=1)
    jumps_before = [len(full.jumps(i)[0]) for i in range(n)]
    full.run_periods(2, is_obs=1, dump_at=[2], dump_base=1)
    a = make(q, P, R, n, 5)
    a.run_periods(3, is_obs=1)
    blob = a.checkpoint()
    a.close()
    b = make(q, P, R, n, 5)  # same configuration (the Philox key is part of it), other states:
    b.run_periods(1, is_obs=0)  # everything the continuation needs comes from the blob
    b.restore(blob)
    b.run_periods(2, is_obs=1, dump_at=[2], dump_base=1)
    for x, y in zip(full.states(), b.states()):
        assert np.array_equal(x, y)
    for i in range(n):
        tf, kf, nf, ef = full.jumps(i)
        tb, kb, nb, eb = b.jumps(i)
        k = jumps_before[i]
        assert np.array_equal(tf[k:], tb) and np.array_equal(kf[k:], kb) and np.array_equal(ef[k:], eb)
    of, ob = full.observables(1, 1, want_adr=True), b.observables(1, 1, want_adr=True)
    for key in of:
        assert np.array_equal(of[key], ob[key]), key


def test_checkpoint_carries_lyapunov_pairs():
    import os_d_b200 as q

    cfg = dict(CFGS[0])
    P = dimer_problem(16, deep=10)
    n, T = 16, P["T"]

    def start():
        e = q.Engine(P["U"], P["L"], [1.0], P["HE"], None, T, n, seed=4, record=1, max_dumps=1)
        e.set_states(start_states(n, P["d"]))
        e.init_thresholds()
        e.set_active(n // 2)
        e.run_periods(1, is_obs=0)
        e.set_active(n)
        e.lpn_start(**cfg)
        e.reset_times()
        return e

    full = start()
    for p in range(4):
        full.run_periods(1)
        full.lpn_period((p + 1) * T)
    a = start()
    for p in range(2):
        a.run_periods(1)
        a.lpn_period((p + 1) * T)
    blob = a.checkpoint()
    b = start()
    b.restore(blob)
    for p in range(2, 4):
        b.run_periods(1)
        b.lpn_period((p + 1) * T)
    assert np.array_equal(full.states()[0], b.states()[0])
    vf, vb = full.lpn_values(), b.lpn_values()
    for key in vf:
        assert np.array_equal(vf[key], vb[key]), key
    assert vf["num_renorms"].sum() > 0
