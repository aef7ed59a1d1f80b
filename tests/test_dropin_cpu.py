"""Parameter files, file-name suffix and error exits of the drop-in executable (no GPU)."""
import os
import subprocess

import pytest

import os_d_b200 as q
from tests.dropin_expect import (BASE_CONFIG, BASE_PARAMS, DIMERSYNC_PARAMS, FLOQ2_PARAMS, FLOQN_PARAMS, FLOQP_PARAMS,
                                 INTEGRABLE_PARAMS, JCS_PARAMS, LPN_PARAMS, MBL_PARAMS, PS_PARAMS, config_text, params_text,
                                 suffix)

EXE = os.path.join(os.path.dirname(q.__file__), "qjx_b200")


def check(tmp_path, cfg, prm, extra_cfg=""):
    (tmp_path / "config.txt").write_text(config_text(cfg) + extra_cfg)
    (tmp_path / "params.txt").write_text(params_text(prm))
    return subprocess.run([EXE, "--check"], cwd=tmp_path, capture_output=True, text=True, timeout=60)


@pytest.mark.parametrize("over", [
    {},
    {"N": 500, "diss_gamma": 0.1, "dimer_drv_ampl": 1.55, "dimer_prm_U": 0.37, "dimer_prm_E": 1.0},
    {"N": 7, "diss_type": 1, "diss_phase": 0.25, "dimer_drv_type": 1, "dimer_drv_freq": 2.5, "dimer_prm_J": -1.25,
     "start_type": 1, "start_state": 3},
])
def test_suffix_matches_reference_rule(tmp_path, over):
    prm = dict(BASE_PARAMS, **over)
    r = check(tmp_path, BASE_CONFIG, prm)
    assert r.returncode == 0, r.stdout
    line = [x for x in r.stdout.splitlines() if x.startswith("fn_suffix = ")][0]
    assert line[len("fn_suffix = "):] == suffix(BASE_CONFIG, prm)


def test_config_parsing_rules(tmp_path):
    # lines with a number of tokens other than two are ignored; last value wins; CR tolerated
    extra = "seed 11 12\nnum_trajectories 5\r\nmns\nseed 9\n"
    r = check(tmp_path, BASE_CONFIG, BASE_PARAMS, extra)
    assert r.returncode == 0
    assert "seed = 9" in r.stdout and "num_trajectories = 5" in r.stdout and "mns = 1000000" in r.stdout
    assert "_rnd(9_1000000)" in r.stdout


def test_params_echo_format(tmp_path):
    r = check(tmp_path, BASE_CONFIG, BASE_PARAMS)
    assert r.stdout.startswith("############# parameters #############\nsys_id = 0\ntask_id = 1\nprop_id = 0\n")
    assert "diss_gamma: 0.1\n" in r.stdout and "N: 16\n" in r.stdout


@pytest.mark.parametrize("over", [{}, {"lpn_type": -1, "lpn_delta_s": 2.5e-4, "lpn_delta_f_high": 0.3,
                                      "lpn_delta_f_low": 3e-6}, {"lpn_type": -2}])
def test_lpn_suffix_matches_reference_rule(tmp_path, over):
    """LpnMult appends suffix_lpn (outputter.cpp:34-38, 371-381)."""
    cfg = dict(BASE_CONFIG, task_id=7)
    prm = {**BASE_PARAMS, **LPN_PARAMS, **over}
    r = check(tmp_path, cfg, prm)
    assert r.returncode == 0, r.stdout
    line = [x for x in r.stdout.splitlines() if x.startswith("fn_suffix = ")][0]
    assert line[len("fn_suffix = "):] == suffix(cfg, prm) and "_lpn(" in line


@pytest.mark.parametrize("over", [{}, {"jcs_drv_part_1": 1.25, "jcs_drv_ampl": 0.05, "diss_type": 1}])
def test_jcs_suffix_matches_reference_rule(tmp_path, over):
    """JCSOutputBehavior::suffix_param (outputter.cpp:95-133)."""
    cfg = dict(BASE_CONFIG, sys_id=1)
    prm = {**BASE_PARAMS, **JCS_PARAMS, **over}
    r = check(tmp_path, cfg, prm)
    assert r.returncode == 0, r.stdout
    line = [x for x in r.stdout.splitlines() if x.startswith("fn_suffix = ")][0]
    assert line[len("fn_suffix = "):] == suffix(cfg, prm) and "_prm(5.0000)" in line


@pytest.mark.parametrize("over", [{}, {"diss_type": 0, "diss_phase": 0.125, "mbl_seed": 17, "mbl_prm_W": 12.0}])
def test_mbl_suffix_matches_reference_rule(tmp_path, over):
    """MBLOutputBehavior::suffix_param (outputter.cpp:176-212): a second _rnd() with the disorder
    stream, and diss() in the order type, phase, gamma."""
    cfg = dict(BASE_CONFIG, sys_id=3)
    prm = {**BASE_PARAMS, **MBL_PARAMS, **over}
    r = check(tmp_path, cfg, prm)
    assert r.returncode == 0, r.stdout
    line = [x for x in r.stdout.splitlines() if x.startswith("fn_suffix = ")][0]
    assert line[len("fn_suffix = "):] == suffix(cfg, prm) and "_Nc(8)_rnd(" in line


@pytest.mark.parametrize("sys_id,task_id,prop_id", [(3, 4, 0), (1, 4, 0), (3, 7, 1), (1, 1, 1), (5, 4, 0), (2, 7, 0),
                                                     (6, 8, 0), (6, 1, 1)])
def test_jcs_mbl_other_tasks_exit_with_error(tmp_path, sys_id, task_id, prop_id):
    prm = {**BASE_PARAMS, **LPN_PARAMS, **SYS_PARAMS[sys_id]}
    r = check(tmp_path, dict(BASE_CONFIG, sys_id=sys_id, task_id=task_id, prop_id=prop_id), prm)
    assert r.returncode != 0 and "Error: Wrong task_id / prop_id for sys_id %d" % sys_id in r.stdout


def test_lpn_mult_deep_checks(tmp_path):
    """LpnMultDeep (task_id 8) appends suffix_lpn, runs the dimer with the QJ propagator only."""
    cfg = dict(BASE_CONFIG, task_id=8)
    prm = {**BASE_PARAMS, **LPN_PARAMS, "deep_num_steps": 2}
    r = check(tmp_path, cfg, prm)
    assert r.returncode == 0, r.stdout
    line = [x for x in r.stdout.splitlines() if x.startswith("fn_suffix = ")][0]
    assert line[len("fn_suffix = "):] == suffix(cfg, prm) and "_setup(0_8_0)" in line
    r = check(tmp_path, dict(cfg, prop_id=1), prm)
    assert r.returncode != 0 and "Error: Wrong prop_id" in r.stdout
    r = check(tmp_path, dict(cfg, sys_id=1), {**prm, **JCS_PARAMS})
    assert r.returncode != 0 and "Error: Wrong task_id / prop_id for sys_id 1" in r.stdout


SYS_PARAMS = {1: JCS_PARAMS, 2: PS_PARAMS, 3: MBL_PARAMS, 5: INTEGRABLE_PARAMS, 6: DIMERSYNC_PARAMS, 7: FLOQ2_PARAMS,
              8: FLOQN_PARAMS, 9: FLOQP_PARAMS}


@pytest.mark.parametrize("sys_id,task_id", [(1, 7), (3, 7), (5, 7), (5, 1), (2, 1), (6, 1), (6, 7), (7, 1), (7, 7),
                                            (8, 1), (8, 7), (9, 1), (9, 7)])
def test_jcs_mbl_integrable_suffix(tmp_path, sys_id, task_id):
    """suffix_param (+ suffix_lpn for LpnMult) of JCS, MBL and Integrable (outputter.cpp:95-269,
    371-381); Integrable prints tau and k as integers."""
    cfg = dict(BASE_CONFIG, sys_id=sys_id, task_id=task_id)
    prm = {**BASE_PARAMS, **LPN_PARAMS, **SYS_PARAMS[sys_id]}
    r = check(tmp_path, cfg, prm)
    assert r.returncode == 0, r.stdout
    line = [x for x in r.stdout.splitlines() if x.startswith("fn_suffix = ")][0]
    assert line[len("fn_suffix = "):] == suffix(cfg, prm) and ("_lpn(" in line) == (task_id == 7)


@pytest.mark.parametrize("key,val", [("sys_id", 4), ("sys_id", 10), ("task_id", 9), ("prop_id", 2)])
def test_unsupported_ids_exit_with_error(tmp_path, key, val):
    r = check(tmp_path, dict(BASE_CONFIG, **{key: val}), BASE_PARAMS)
    assert r.returncode != 0 and "Error: Wrong " + key in r.stdout


def test_missing_param_is_an_error(tmp_path):
    prm = dict(BASE_PARAMS)
    del prm["diss_gamma"]
    r = check(tmp_path, BASE_CONFIG, prm)
    assert r.returncode != 0 and "missing key in params file: diss_gamma" in r.stdout


def test_missing_files_use_defaults(tmp_path):
    r = subprocess.run([EXE, "--check"], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert "Unable to open file" in r.stdout and "Init with default params" in r.stdout
    assert r.returncode != 0  # default task_id 0 is not the Std task


def test_config_tokenisation_edge_cases(tmp_path):
    """Only the single space separates tokens, runs of spaces and spaces at either end make no
    token, and a tab stays inside its token (so such a line has one token and is ignored)."""
    extra = "seed\t5\n  mns   77  \n num_trajectories  7 \n  \nex_deep 12 \t\n"
    r = check(tmp_path, BASE_CONFIG, BASE_PARAMS, extra)
    assert r.returncode == 0, r.stdout
    assert "mns = 77" in r.stdout and "num_trajectories = 7" in r.stdout
    assert "seed = 5" not in r.stdout
    # "ex_deep 12 \t" has the tokens "ex_deep", "12" and "\t": three tokens, ignored
    assert "ex_deep = 12" not in r.stdout
