"""The drop-in executable (os_d_b200/qjx_b200) on a GPU, compared file by file with the
reference's Std-task outputs computed by the CPU oracle on the same inputs."""
import copy
import math
import os
import subprocess

import pytest

import os_d_b200 as q
from tests.dropin_expect import (BASE_CONFIG, BASE_PARAMS, DIMERSYNC_PARAMS, FLOQ2_PARAMS, FLOQN_PARAMS, FLOQP_PARAMS,
                                 INTEGRABLE_PARAMS, JCS_PARAMS, LPN_PARAMS, MBL_PARAMS, PS_PARAMS, config_text,
                                 expected_outputs, params_text)

pytestmark = pytest.mark.gpu
EXE = os.path.join(os.path.dirname(q.__file__), "qjx_b200")


def run_case(tmp_path, cfg, prm):
    (tmp_path / "config.txt").write_text(config_text(cfg))
    (tmp_path / "params.txt").write_text(params_text(prm))
    if cfg.get("path"):
        (tmp_path / cfg["path"]).mkdir(parents=True, exist_ok=True)
    r = subprocess.run([EXE], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    d = int(prm["N"]) + 1
    d = int(prm["N"]) if cfg.get("sys_id", 0) == 1 else d
    d = math.comb(int(prm["mbl_Nc"]), int(prm["mbl_Nc"]) // 2) if cfg.get("sys_id", 0) == 3 else d
    d = 1 << int(prm["integrable_N"]) if cfg.get("sys_id", 0) == 5 else d
    d = (1 << int(prm["ps_num_spins"])) * int(prm["ps_num_photons_states"]) if cfg.get("sys_id", 0) == 2 else d
    d = int(prm["dimersync_N"]) + 1 if cfg.get("sys_id", 0) == 6 else d
    d = 4 if cfg.get("sys_id", 0) == 7 else d
    d = 1 << int(prm["flqnsp_n"]) if cfg.get("sys_id", 0) == 8 else d
    d = 2 * (int(prm["flq_sp_ph_n_ph"]) + 1) if cfg.get("sys_id", 0) == 9 else d
    R = q.random_observables(d, int(prm["num_random_obs"]), int(prm["random_obs_seed"]),
                             int(prm["random_obs_mns"]), int(prm["random_obs_type"]))
    exp = expected_outputs(cfg, prm, R)
    written = set()
    for root, _, names in os.walk(tmp_path):
        for nm in names:
            rel = os.path.relpath(os.path.join(root, nm), tmp_path)
            if rel not in ("config.txt", "params.txt"):
                written.add(rel)
    assert written == set(exp), (sorted(written ^ set(exp)))[:10]
    for name, text in exp.items():
        got = (tmp_path / name).read_text()
        assert got == text, name
    return exp


def test_std_task_files_match(tmp_path):
    exp = run_case(tmp_path, BASE_CONFIG, BASE_PARAMS)
    assert any(k.startswith("jump_times_") for k in exp)


def test_per_dump_files_log_dumps_and_debug(tmp_path):
    cfg = dict(BASE_CONFIG, is_debug=1, is_pp=1, num_obs_periods=20, path="out/")
    prm = dict(BASE_PARAMS, dump_type=1, dump_num=4, dump_phi=1, dump_phi_evo=1, dump_adr_sep=1, dump_adr_avg=1,
               dump_evo_avg=1, num_random_obs=2, start_type=1)
    run_case(tmp_path, cfg, prm)


def test_early_stop_on_jump_counts(tmp_path):
    cfg = dict(BASE_CONFIG, num_obs_periods=40, num_trajectories=6)
    prm = dict(BASE_PARAMS, dump_num=4, jump=1, jumps_counts=5, dump_adr_avg=1, num_random_obs=0)
    run_case(tmp_path, cfg, prm)


def test_dims_101_sample(tmp_path):
    cfg = dict(BASE_CONFIG, num_trajectories=16, num_tp_periods=1, num_obs_periods=2, seed=42)
    prm = dict(BASE_PARAMS, N=100, dump_num=2, jump=2)
    run_case(tmp_path, cfg, prm)


def test_purity_per_dump(tmp_path):
    cfg = dict(BASE_CONFIG, num_obs_periods=6, num_trajectories=24)
    prm = dict(BASE_PARAMS, dump_num=3, dump_purity=1)
    exp = run_case(tmp_path, cfg, prm)
    vals = [float(v) for k, t in exp.items() if k.startswith("purity_evo") for v in t.split()]
    assert len(vals) == 4 and 0.0 < min(vals) <= max(vals) < 1.0  # dump 0 follows the transient periods


def test_rk_propagator_files_match(tmp_path):
    cfg = dict(BASE_CONFIG, prop_id=1, rk_ns=400, num_tp_periods=1, num_obs_periods=3, num_trajectories=12,
               is_debug=1)
    prm = dict(BASE_PARAMS, dump_num=3, jump=2)
    exp = run_case(tmp_path, cfg, prm)
    assert any(k.startswith("jump_times_") and exp[k] for k in exp)


def test_std_deep_task_files_match(tmp_path):
    cfg = dict(BASE_CONFIG, task_id=4, num_tp_periods=1, num_obs_periods=2, num_trajectories=10, is_debug=1)
    prm = dict(BASE_PARAMS, deep_num_steps=2, dump_adr_sep=1, dump_adr_avg=1, dump_evo_avg=1, jump=2)
    exp = run_case(tmp_path, cfg, prm)
    assert any(k.startswith("adr_0") for k in exp)


def test_lpn_mult_task_files_match(tmp_path):
    """LpnMult (task_id 7), random-observable distance, renormalisation on the thresholds, the
    save_lambdas records and the adr files."""
    cfg = dict(BASE_CONFIG, task_id=7, num_trajectories=12, num_tp_periods=2, num_obs_periods=6)
    prm = {**BASE_PARAMS, **LPN_PARAMS, "dump_num": 3, "lpn_delta_f_high": 5e-3, "lpn_delta_f_low": 5e-4,
           "save_lambdas": 1, "dump_adr_sep": 1, "dump_adr_avg": 1}
    exp = run_case(tmp_path, cfg, prm)
    assert any(k.startswith("deltas_s_") and exp[k] for k in exp)
    assert any(k.startswith("lambda_evo") for k in exp)


def test_lpn_mult_every_period_rk(tmp_path):
    """LpnMult with lambda_lpn_now (every period), the mean distance, the RK propagator,
    logarithmic dumps and the per-dump adr average over the bases."""
    cfg = dict(BASE_CONFIG, task_id=7, prop_id=1, rk_ns=400, num_trajectories=8, num_tp_periods=1,
               num_obs_periods=5, is_pp=1)
    prm = {**BASE_PARAMS, **LPN_PARAMS, "lpn_type": -1, "lambda_per_periods": 1, "dump_type": 1, "dump_num": 2,
           "dump_evo_avg": 1, "dump_adr_avg": 1, "num_random_obs": 2}
    run_case(tmp_path, cfg, prm)


@pytest.mark.parametrize("diss_type", [1, 0])
def test_mbl_system_files_match(tmp_path, diss_type):
    """The MBL system (sys_id 3): 70 basis words of 8 cells, 7 hop-dissipators (diss_type 1) or 8
    occupation dissipators (diss_type 0), spec = <H> / W and the imbalance from the adr rows
    (newdel.cpp:182-271, 868-958, 1699-1815, 2751-2838; experiment.cpp:1705-1800; core.cpp:4190-5056)."""
    cfg = dict(BASE_CONFIG, sys_id=3, num_trajectories=16, num_tp_periods=1, num_obs_periods=4, is_debug=1)
    prm = {**BASE_PARAMS, **MBL_PARAMS, "diss_type": diss_type, "dump_num": 2, "jump": 2, "dump_adr_sep": 1,
           "dump_adr_avg": 1, "start_state": 5}
    exp = run_case(tmp_path, cfg, prm)
    assert any(k.startswith("imbalance_evo") for k in exp) and any(k.startswith("energies") for k in exp)
    types = set()
    for k, v in exp.items():
        if k.startswith("diss_types_"):
            types.update(int(x) for x in v.split())
    assert len(types) > 3  # several channels chosen


@pytest.mark.parametrize("lpn_type", [-1, -2, 0])
def test_mbl_lpn_mult_files_match(tmp_path, lpn_type):
    """MBL LpnMult (sys_id 3, task_id 7; the production MBL sweeps, submit_mbl.py): spec, imbalance
    and random-observable distances, the MBL file set (core.cpp:4910-5096) incl. save_lambdas."""
    cfg = dict(BASE_CONFIG, sys_id=3, task_id=7, num_trajectories=16, num_tp_periods=2, num_obs_periods=5)
    prm = {**BASE_PARAMS, **LPN_PARAMS, **MBL_PARAMS, "lpn_type": lpn_type, "dump_num": 5, "jump": 1,
           "dump_adr_sep": 1, "dump_adr_avg": 1, "save_lambdas": 1, "lpn_delta_f_high": 1e-2}
    exp = run_case(tmp_path, cfg, prm)
    k = [k for k in exp if k.startswith("num_renorms")][0]
    assert sum(int(x) for x in exp[k].split()) > 0  # renormalisations happened
    assert any(k.startswith("imbalance_lpn_evo") for k in exp) and any(k.startswith("spec_lpn_evo") for k in exp)


@pytest.mark.parametrize("lpn_type", [-1, -2, 0])
def test_jcs_lpn_mult_files_match(tmp_path, lpn_type):
    """JCS LpnMult (sys_id 1, task_id 7; submit_jcs.py): spec = <a> / alpha, <a^+ a> / d and
    random-observable distances, Lyapunov time in units of calc_T = (part_1 + part_2) alpha, adr rows
    left as the std ones (JCS's calc_chars_lpn does not rewrite them), the JCS file set
    (core.cpp:2976-3150)."""
    cfg = dict(BASE_CONFIG, sys_id=1, task_id=7, num_trajectories=16, num_tp_periods=2, num_obs_periods=5)
    prm = {**BASE_PARAMS, **LPN_PARAMS, **JCS_PARAMS, "lpn_type": lpn_type, "dump_num": 5, "jump": 1,
           "dump_adr_sep": 1, "dump_adr_avg": 1, "save_lambdas": 1, "lpn_delta_f_high": 1e-2}
    exp = run_case(tmp_path, cfg, prm)
    k = [k for k in exp if k.startswith("num_renorms")][0]
    assert sum(int(x) for x in exp[k].split()) > 0
    assert any(k.startswith("mean_lpn_evo") for k in exp) and any(k.startswith("spec_lpn_evo") for k in exp)


@pytest.mark.parametrize("diss_type,spins", [(1, 1), (0, 2)])
def test_ps_system_files_match(tmp_path, diss_type, spins):
    """The PS system (sys_id 2): spins x photons, kick and free evolution each run as two halves,
    spec = <a> / alpha, spec_2 = <J_z>, spec_3 = <J_+>, mean = <a^+ a> (newdel.cpp:132-181, 650-866,
    1582-1697, 2603-2749; core.cpp:3245-4130, 10234-10305)."""
    cfg = dict(BASE_CONFIG, sys_id=2, num_trajectories=16, num_tp_periods=1, num_obs_periods=4, is_debug=1)
    prm = {**BASE_PARAMS, **PS_PARAMS, "diss_type": diss_type, "ps_num_spins": spins, "dump_num": 2, "jump": 2,
           "dump_adr_sep": 1, "dump_adr_avg": 1}
    exp = run_case(tmp_path, cfg, prm)
    assert any(k.startswith("spec_3_evo") for k in exp)


def test_integrable_system_files_match(tmp_path):
    """The Integrable system (sys_id 5): 6 spins (d = 64), H = 0, 6 pair dissipators incl. the
    border, spec = <special> (newdel.cpp:310-345, 1030-1095, 1924-2076, 2914-3004; core.cpp:6470-6819)."""
    cfg = dict(BASE_CONFIG, sys_id=5, num_trajectories=16, num_tp_periods=1, num_obs_periods=4, is_debug=1)
    prm = {**BASE_PARAMS, **INTEGRABLE_PARAMS, "dump_num": 2, "jump": 2, "dump_adr_sep": 1, "dump_adr_avg": 1}
    exp = run_case(tmp_path, cfg, prm)
    types = set()
    for k, v in exp.items():
        if k.startswith("diss_types_"):
            types.update(int(x) for x in v.split())
    assert len(types) == 6


@pytest.mark.parametrize("lpn_type", [-1, 0])
def test_integrable_lpn_mult_files_match(tmp_path, lpn_type):
    """Integrable LpnMult (sys_id 5, task_id 7; submit_integrable.py): spec and random-observable
    distances, the Integrable Lyapunov file set (core.cpp:6685-6858)."""
    cfg = dict(BASE_CONFIG, sys_id=5, task_id=7, num_trajectories=16, num_tp_periods=2, num_obs_periods=5)
    prm = {**BASE_PARAMS, **LPN_PARAMS, **INTEGRABLE_PARAMS, "lpn_type": lpn_type, "dump_num": 5, "jump": 1,
           "dump_adr_sep": 1, "dump_adr_avg": 1, "save_lambdas": 1, "lpn_delta_f_high": 1e-2}
    exp = run_case(tmp_path, cfg, prm)
    k = [k for k in exp if k.startswith("num_renorms")][0]
    assert sum(int(x) for x in exp[k].split()) > 0


@pytest.mark.parametrize("per_period", [0, 1])
def test_lpn_mult_deep_files_match(tmp_path, per_period):
    """LpnMultDeep (task_id 8, the dimer): base/variation pairs advanced sub-period by sub-period
    (qjx_run_sub_periods), the Lyapunov step after every sub-period (lambda_per_periods 0) or at the
    last one of each period with the bases' characteristics in between (1), one dump per sub-period
    (experiment.cpp:302-350; core.cpp:155-241)."""
    cfg = dict(BASE_CONFIG, task_id=8, num_trajectories=12, num_tp_periods=1, num_obs_periods=2)
    prm = {**BASE_PARAMS, **LPN_PARAMS, "deep_num_steps": 2, "lambda_per_periods": per_period, "jump": 1,
           "dump_adr_sep": 1, "dump_adr_avg": 1, "dump_evo_avg": 1, "save_lambdas": 1, "lpn_delta_f_high": 1e-2,
           "dump_phi_evo": 1}
    exp = run_case(tmp_path, cfg, prm)
    k = [k for k in exp if k.startswith("num_renorms")][0]
    assert sum(int(x) for x in exp[k].split()) > 0


@pytest.mark.parametrize("task_id", [1, 7])
def test_dimersync_files_match(tmp_path, task_id):
    """DimerSync (sys_id 6): the dimer's QJ branches under the dimersync_* keys, drive 1 in the
    branches and drive 2's period (newdel.cpp:39-95, 500-563, 2390-2498; core.cpp:9983-10030)."""
    cfg = dict(BASE_CONFIG, sys_id=6, task_id=task_id, num_trajectories=12, num_tp_periods=1, num_obs_periods=4)
    prm = {**BASE_PARAMS, **LPN_PARAMS, **DIMERSYNC_PARAMS, "dump_num": 4, "jump": 1, "dump_adr_sep": 1,
           "lpn_delta_f_high": 1e-2}
    run_case(tmp_path, cfg, prm)


@pytest.mark.parametrize("task_id,is_debug", [(1, 1), (7, 0)])
def test_floq2spins_files_match(tmp_path, task_id, is_debug):
    """Floq2Spins (sys_id 7): two spins, sigma_- on each, the undriven QJ branch covering T / 2 per
    period, spec = <H> (newdel.cpp:346-378, 1096-1182, 2077-2136, 3005-3101; core.cpp:6865-7830)."""
    cfg = dict(BASE_CONFIG, sys_id=7, task_id=task_id, num_trajectories=16, num_tp_periods=1, num_obs_periods=4,
               is_debug=is_debug)
    prm = {**BASE_PARAMS, **LPN_PARAMS, **FLOQ2_PARAMS, "dump_num": 4, "jump": 2, "dump_adr_sep": 1,
           "lpn_delta_f_high": 1e-2}
    run_case(tmp_path, cfg, prm)


@pytest.mark.parametrize("task_id,is_debug", [(1, 1), (7, 0)])
def test_floqnspins_files_match(tmp_path, task_id, is_debug):
    """FloqManySpins (sys_id 8): 3 spins, H = (Delta/2) sum sz + J sy sy sy (imaginary), sigma_- on
    each spin, the undriven QJ branch (newdel.cpp:379-413, 1184-1332, 2138-2224, 3103-3199)."""
    cfg = dict(BASE_CONFIG, sys_id=8, task_id=task_id, num_trajectories=16, num_tp_periods=1, num_obs_periods=4,
               is_debug=is_debug)
    prm = {**BASE_PARAMS, **LPN_PARAMS, **FLOQN_PARAMS, "dump_num": 4, "jump": 2, "dump_adr_sep": 1,
           "lpn_delta_f_high": 1e-2}
    run_case(tmp_path, cfg, prm)


@pytest.mark.parametrize("task_id,is_debug", [(1, 1), (7, 0)])
def test_floqspph_files_match(tmp_path, task_id, is_debug):
    """FloqSpinPh (sys_id 9): a spin and 9 photon states, photon loss a, the undriven QJ branch
    (newdel.cpp:414-449, 1334-1452, 2226-2284, 3201-3297)."""
    cfg = dict(BASE_CONFIG, sys_id=9, task_id=task_id, num_trajectories=16, num_tp_periods=1, num_obs_periods=4,
               is_debug=is_debug)
    prm = {**BASE_PARAMS, **LPN_PARAMS, **FLOQP_PARAMS, "dump_num": 4, "jump": 2, "dump_adr_sep": 1,
           "lpn_delta_f_high": 1e-2, "start_state": 16}
    run_case(tmp_path, cfg, prm)


def test_jcs_system_files_match(tmp_path):
    """The JCS system (sys_id 1): kick and free evolution of unequal duration, spec = <a> / alpha,
    mean = <a^+ a> (newdel.cpp:96-130, 564-649, 1546-1580, 2499-2601; core.cpp:2739-3102)."""
    cfg = dict(BASE_CONFIG, sys_id=1, num_trajectories=16, num_tp_periods=1, num_obs_periods=4, is_debug=1)
    prm = {**BASE_PARAMS, **JCS_PARAMS, "dump_num": 2, "jump": 2, "dump_adr_sep": 1, "dump_adr_avg": 1}
    exp = run_case(tmp_path, cfg, prm)
    assert any(k.startswith("spec_evo") for k in exp) and any(k.startswith("jump_times_") and exp[k] for k in exp)
