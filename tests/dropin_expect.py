"""Expected output files of the drop-in executable, computed with the CPU oracle.

Replays the reference's Std task with the QJ propagator (source/cpp/QJX/QJX/experiment.cpp:
411-542, core.cpp:918-1084, dump.cpp:3-61, core.cpp:12567-12613) on the oracle and renders
every file with the reference's formats (source/cpp/QJX/QJX/utils.cpp, utils.h).
"""
import os

import numpy as np

from oracle import oracle_py as O

TWO_PI = 2.0 * 3.1415926535897932384626433832795


def write_files(d, files):
    for name, text in files.items():
        with open(os.path.join(d, name), "w") as f:
            f.write(text)


def config_text(cfg):
    return "".join(f"{k} {v}\n" for k, v in cfg.items())


def params_text(prm):
    return "".join(f"{k} {v}\n" for k, v in prm.items())


def fmt_double(x):
    return "%.16e" % x


def f_double_data(v):
    return "".join(fmt_double(x) + "\n" for x in v)


def f_int_data(v):
    return "".join("%d\n" % x for x in v)


def f_complex_data(v):
    return "".join(fmt_double(z.real) + " " + fmt_double(z.imag) + "\n" for z in v)


def f_2d_inv(rows_by_cols):  # array [rows][cols]
    return "".join("".join(fmt_double(x) + " " for x in row) + "\n" for row in rows_by_cols)


def f_2d_inv_complex(rows_by_cols):  # save_2d_inv_complex_data: "re im " pairs, rows = dumps
    return "".join("".join(fmt_double(z.real) + " " + fmt_double(z.imag) + " " for z in row) + "\n"
                   for row in rows_by_cols)


def f_2d_complex(rows_by_cols):
    return "".join("\t".join("(%s,%s)" % (fmt_double(z.real), fmt_double(z.imag)) for z in row) + "\n"
                   for row in rows_by_cols)


def suffix(cfg, prm):
    """DimerOutputBehavior::suffix_param with precision 4 (outputter.cpp:3-44, 353-388);
    JCSOutputBehavior::suffix_param for sys_id 1 (outputter.cpp:95-133); MBLOutputBehavior::suffix_param
    for sys_id 3 (outputter.cpp:176-212)."""
    f4 = lambda x: format(float(x), "0.4f")  # noqa: E731
    if cfg.get("sys_id", 0) == 9:  # FloqSpinPhOutputBehavior::suffix_param (outputter.cpp:326-353)
        return ("_setup(%d_%d_%d)" % (9, cfg.get("task_id", 0), cfg.get("prop_id", 0))
                + "_rnd(%d_%d)" % (cfg.get("seed", 0), cfg.get("mns", 1000000))
                + "_nph(%d)" % int(prm["flq_sp_ph_n_ph"])
                + "".join("_%s(%s)" % (k, f4(prm[key])) for k, key in (
                    ("ampl", "flq_sp_ph_ampl"), ("freq", "flq_sp_ph_freq"), ("D", "flq_sp_ph_Delta"),
                    ("O", "flq_sp_ph_Omega"), ("gamma", "flq_sp_ph_gamma")))
                + (lpn_suffix(prm) if cfg.get("task_id", 0) in (7, 8) else "") + ".txt")
    if cfg.get("sys_id", 0) == 8:  # FloqManySpinsOutputBehavior::suffix_param (outputter.cpp:299-326)
        return ("_setup(%d_%d_%d)" % (8, cfg.get("task_id", 0), cfg.get("prop_id", 0))
                + "_rnd(%d_%d)" % (cfg.get("seed", 0), cfg.get("mns", 1000000))
                + "_n(%d)" % int(prm["flqnsp_n"])
                + "".join("_%s(%s)" % (k, f4(prm[key])) for k, key in (
                    ("ampl", "flqnsp_ampl"), ("freq", "flqnsp_freq"), ("D", "flqnsp_Delta"), ("J", "flqnsp_J"),
                    ("gamma", "flqnsp_gamma")))
                + (lpn_suffix(prm) if cfg.get("task_id", 0) in (7, 8) else "") + ".txt")
    if cfg.get("sys_id", 0) == 7:  # Floq2SpinsOutputBehavior::suffix_param (outputter.cpp:271-299)
        return ("_setup(%d_%d_%d)" % (7, cfg.get("task_id", 0), cfg.get("prop_id", 0))
                + "_rnd(%d_%d)" % (cfg.get("seed", 0), cfg.get("mns", 1000000))
                + "".join("_%s(%s)" % (k, f4(prm[key])) for k, key in (
                    ("ampl", "flq2sp_ampl"), ("freq", "flq2sp_freq"), ("D1", "flq2sp_Delta_1"), ("D2", "flq2sp_Delta_2"),
                    ("J", "flq2sp_J"), ("gamma", "flq2sp_gamma")))
                + (lpn_suffix(prm) if cfg.get("task_id", 0) in (7, 8) else "") + ".txt")
    if cfg.get("sys_id", 0) == 6:  # DimerSyncOutputBehavior::suffix_param (outputter.cpp:45-93)
        return ("_setup(%d_%d_%d)" % (6, cfg.get("task_id", 0), cfg.get("prop_id", 0))
                + "_rnd(%d_%d)" % (cfg.get("seed", 0), cfg.get("mns", 1000000))
                + "_N(%d)" % int(prm["dimersync_N"])
                + "_diss(%d_%s_%s)" % (int(prm["diss_type"]), f4(prm["diss_gamma"]), f4(prm["diss_phase"]))
                + "".join("_drv%d(%s_%s_%s)" % (i, f4(prm["dimersync_drv_ampl_%d" % i]),
                                                f4(prm["dimersync_drv_freq_%d" % i]), f4(prm["dimersync_drv_phase_%d" % i]))
                          for i in (1, 2))
                + "_T(%d)" % int(prm["dimersync_main_period"])
                + "_prm(%s_%s_%s)" % (f4(prm["dimersync_prm_E"]), f4(prm["dimersync_prm_U"]), f4(prm["dimersync_prm_J"]))
                + "_start(%d_%d)" % (int(prm["start_type"]), int(prm["start_state"]))
                + (lpn_suffix(prm) if cfg.get("task_id", 0) in (7, 8) else "") + ".txt")
    if cfg.get("sys_id", 0) == 2:  # PSOutputBehavior::suffix_param (outputter.cpp:135-174)
        return ("_setup(%d_%d_%d)" % (2, cfg.get("task_id", 0), cfg.get("prop_id", 0))
                + "_rnd(%d_%d)" % (cfg.get("seed", 0), cfg.get("mns", 1000000))
                + "_s(%d)_nps(%d)" % (int(prm["ps_num_spins"]), int(prm["ps_num_photons_states"]))
                + "_diss(%d_%s)" % (int(prm["diss_type"]), f4(prm["ps_diss_w"]))
                + "_drv(%s_%s_%s)" % (f4(prm["ps_drv_part_1"]), f4(prm["ps_drv_part_2"]), f4(prm["ps_drv_ampl"]))
                + "_prm(%s_%s_%s)" % (f4(prm["ps_prm_alpha"]), f4(prm["ps_prm_d"]), f4(prm["ps_prm_g"]))
                + "_start(%d_%d)" % (int(prm["start_type"]), int(prm["start_state"]))
                + (lpn_suffix(prm) if cfg.get("task_id", 0) in (7, 8) else "") + ".txt")
    if cfg.get("sys_id", 0) == 5:  # IntegrableOutputBehavior::suffix_param (outputter.cpp:244-269)
        return ("_setup(%d_%d_%d)" % (5, cfg.get("task_id", 0), cfg.get("prop_id", 0))
                + "_rnd(%d_%d)" % (cfg.get("seed", 0), cfg.get("mns", 1000000))
                + "_N(%d)_seed(%d)_tau(%d)_k(%d)" % (int(prm["integrable_N"]), int(prm["integrable_seed"]),
                                                     int(prm["integrable_tau"]), int(prm["integrable_k"]))
                + "_T(%s)" % f4(prm["integrable_T"])
                + (lpn_suffix(prm) if cfg.get("task_id", 0) in (7, 8) else "") + ".txt")
    if cfg.get("sys_id", 0) == 3:
        return ("_setup(%d_%d_%d)" % (3, cfg.get("task_id", 0), cfg.get("prop_id", 0))
                + "_rnd(%d_%d)" % (cfg.get("seed", 0), cfg.get("mns", 1000000))
                + "_Nc(%d)" % int(prm["mbl_Nc"])
                + "_rnd(%d_%d)" % (int(prm["mbl_seed"]), int(prm["mbl_mns"]))
                + "_diss(%d_%s_%s)" % (int(prm["diss_type"]), f4(prm["diss_phase"]), f4(prm["diss_gamma"]))
                + "_prm(%s_%s_%s)" % (f4(prm["mbl_prm_W"]), f4(prm["mbl_prm_U"]), f4(prm["mbl_prm_J"]))
                + "_start(%d_%d)" % (int(prm["start_type"]), int(prm["start_state"]))
                + (lpn_suffix(prm) if cfg.get("task_id", 0) in (7, 8) else "") + ".txt")
    if cfg.get("sys_id", 0) == 1:
        return ("_setup(%d_%d_%d)" % (1, cfg.get("task_id", 0), cfg.get("prop_id", 0))
                + "_rnd(%d_%d)" % (cfg.get("seed", 0), cfg.get("mns", 1000000))
                + "_N(%d)" % int(prm["N"])
                + "_diss(%d_%s_%s)" % (int(prm["diss_type"]), f4(prm["diss_gamma"]), f4(prm["diss_phase"]))
                + "_drv(%s_%s_%s)" % (f4(prm["jcs_drv_part_1"]), f4(prm["jcs_drv_part_2"]), f4(prm["jcs_drv_ampl"]))
                + "_prm(%s)" % f4(prm["jcs_prm_alpha"])
                + "_start(%d_%d)" % (int(prm["start_type"]), int(prm["start_state"]))
                + (lpn_suffix(prm) if cfg.get("task_id", 0) in (7, 8) else "") + ".txt")
    return ("_setup(%d_%d_%d)" % (cfg.get("sys_id", 0), cfg.get("task_id", 0), cfg.get("prop_id", 0))
            + "_rnd(%d_%d)" % (cfg.get("seed", 0), cfg.get("mns", 1000000))
            + "_N(%d)" % int(prm["N"])
            + "_diss(%d_%s_%s)" % (int(prm["diss_type"]), f4(prm["diss_gamma"]), f4(prm["diss_phase"]))
            + "_drv(%d_%s_%s_%s)" % (int(prm["dimer_drv_type"]), f4(prm["dimer_drv_ampl"]),
                                     f4(prm["dimer_drv_freq"]), f4(prm["dimer_drv_phase"]))
            + "_prm(%s_%s_%s)" % (f4(prm["dimer_prm_E"]), f4(prm["dimer_prm_U"]), f4(prm["dimer_prm_J"]))
            + "_start(%d_%d)" % (int(prm["start_type"]), int(prm["start_state"]))
            + (lpn_suffix(prm) if cfg.get("task_id", 0) in (7, 8) else "") + ".txt")


def lpn_suffix(prm):
    """suffix_lpn (outputter.cpp:371-381)."""
    return "_lpn(%g_%.4f_%.4f_%.4f)" % (float(prm["lpn_type"]), np.log10(prm["lpn_delta_s"]),
                                        np.log10(prm["lpn_delta_f_high"]), np.log10(prm["lpn_delta_f_low"]))


def spec_system(cfg, prm, deep):
    """Integrable (sys_id 5) or Floq2Spins (sys_id 7): L, special, H, period T, split trees U, K.
    Integrable: H = 0, a head of duration integrable_T with two children of the same tree;
    Floq2Spins: special = H, one undriven branch covering T / 2 per period (core.cpp:10722-10766)."""
    if cfg.get("sys_id", 0) in (7, 8, 9):  # Floq2Spins, FloqManySpins, FloqSpinPh
        if cfg.get("sys_id", 0) == 9:
            H, L, K = O.floqspph_operators(int(prm["flq_sp_ph_n_ph"]), prm["flq_sp_ph_Delta"], prm["flq_sp_ph_Omega"],
                                           prm["flq_sp_ph_gamma"])
            T = TWO_PI / prm["flq_sp_ph_freq"]
        elif cfg.get("sys_id", 0) == 7:
            H, L, K = O.floq2spins_operators(prm["flq2sp_Delta_1"], prm["flq2sp_Delta_2"], prm["flq2sp_J"],
                                             prm["flq2sp_gamma"])
            T = TWO_PI / prm["flq2sp_freq"]
        else:
            H, L, K = O.floqnspins_operators(int(prm["flqnsp_n"]), prm["flqnsp_Delta"], prm["flqnsp_J"],
                                             prm["flqnsp_gamma"])
            T = TWO_PI / prm["flqnsp_freq"]
        return L, H, H, T, O.split_tree(K, T, deep)[None], K
    L, S, K = integrable_model(prm)
    T = prm["integrable_T"]
    Ut = O.split_tree(K, T, deep)
    return L, S, np.zeros_like(S), T, np.stack([Ut, Ut]), K


def integrable_model(prm):
    """The Integrable operators (L [N], special, K) of a params dict."""
    return O.integrable_operators(int(prm["integrable_N"]), int(prm["integrable_seed"]),
                                  int(prm["integrable_num_seeds"]), float(prm["integrable_tau"]),
                                  float(prm["integrable_k"]))


def dimersync_as_dimer(cfg, prm):
    """DimerSync (sys_id 6) runs the dimer's QJ branches under its own keys (newdel.cpp:39-95,
    500-563, 2390-2498): drive 1, the period of drive dimersync_main_period."""
    if cfg.get("sys_id", 0) != 6:
        return prm
    main = int(prm["dimersync_main_period"])
    return {**prm, "N": prm["dimersync_N"], "dimer_prm_J": prm["dimersync_prm_J"], "dimer_prm_U": prm["dimersync_prm_U"],
            "dimer_prm_E": prm["dimersync_prm_E"], "dimer_drv_ampl": prm["dimersync_drv_ampl_1"],
            "dimer_drv_freq": prm["dimersync_drv_freq_%d" % main]}


def expected_outputs(cfg, prm, R=None):
    """All files the drop-in writes, as {relative file name: text}."""
    if cfg.get("task_id", 1) in (7, 8):
        return expected_lpn_outputs(cfg, prm, R)
    sfx_prm, prm = prm, dimersync_as_dimer(cfg, prm)
    jcs = cfg.get("sys_id", 0) == 1
    mbl = cfg.get("sys_id", 0) == 3
    integ = cfg.get("sys_id", 0) in (5, 7, 8, 9)  # Integrable and the Floquet systems
    ps = cfg.get("sys_id", 0) == 2
    N = 0 if (mbl or integ or ps) else int(prm["N"])
    d = N if jcs else N + 1
    if mbl:
        Nc = int(prm["mbl_Nc"])
        d = len(O.mbl_basis(Nc))
    if integ:
        d = {7: 4, 8: 1 << int(prm.get("flqnsp_n", 0)), 9: 2 * (int(prm.get("flq_sp_ph_n_ph", 0)) + 1)}.get(
            cfg.get("sys_id", 0), 1 << int(prm.get("integrable_N", 0)))
    if ps:
        d = (1 << int(prm["ps_num_spins"])) * int(prm["ps_num_photons_states"])
    n = cfg["num_trajectories"]
    deep = cfg.get("ex_deep", 16)
    seed = cfg.get("seed", 0)
    path = cfg.get("path", "")
    sfx = suffix(cfg, sfx_prm)
    nr = int(prm["num_random_obs"])
    deep_task = cfg.get("task_id", 1) == 4
    nsub = int(prm.get("deep_num_steps", 0)) if deep_task else 0
    if jcs:  # JCS: kick and free evolution of heads part_b * alpha, spec = <a> / alpha, mean = <a^+ a>
        alpha = prm["jcs_prm_alpha"]
        H, Hd, L, Nop, K0, K1 = O.jcs_operators(N, alpha, prm["jcs_drv_ampl"])
        heads = [prm["jcs_drv_part_1"] * alpha, prm["jcs_drv_part_2"] * alpha]
        # each part runs as the head's two children (init_split_structure_jcs, core.cpp:10086-10157)
        U0, U1 = O.split_tree(K0, heads[0], deep), O.split_tree(K1, heads[1], deep)
        U = np.stack([U0, U0, U1, U1])
        HE = Nop
        Rs = np.concatenate([L[None], R]) if nr else L[None]
        T = t_head = alpha
        ens = O.Ensemble(U, L, [1.0], HE, Rs, T, n, seed=seed, record=int(prm["jump"]), rec_cap=100000,
                         branch_len=[0.5 * heads[0], 0.5 * heads[0], 0.5 * heads[1], 0.5 * heads[1]])
    elif ps:  # PS: like JCS with spins; spec, spec_2, spec_3, photons ride in observable slots 0..3
        alpha = prm["ps_prm_alpha"]
        H, Hd, L, S4, K0, K1 = O.ps_operators(int(prm["ps_num_spins"]), int(prm["ps_num_photons_states"]), alpha,
                                              prm["ps_prm_d"], prm["ps_prm_g"], prm["ps_drv_ampl"],
                                              int(prm["diss_type"]), prm["ps_diss_w"])
        heads = [prm["ps_drv_part_1"] * alpha, prm["ps_drv_part_2"] * alpha]
        U0, U1 = O.split_tree(K0, heads[0], deep), O.split_tree(K1, heads[1], deep)
        U = np.stack([U0, U0, U1, U1])
        Rs = np.concatenate([S4, R]) if nr else S4
        T = alpha
        ens = O.Ensemble(U, L, [1.0] * L.shape[0], H, Rs, T, n, seed=seed, record=int(prm["jump"]), rec_cap=100000,
                         branch_len=[0.5 * heads[0], 0.5 * heads[0], 0.5 * heads[1], 0.5 * heads[1]])
    elif integ:  # Integrable / Floq2Spins: spec = <special>
        Ls, S, H, T, U, K = spec_system(cfg, prm, deep)
        Ut = U[0]
        Rs = np.concatenate([S[None], R]) if nr else S[None]
        ens = O.Ensemble(U, Ls, [1.0] * Ls.shape[0], H, Rs, T, n, seed=seed, record=int(prm["jump"]), rec_cap=100000)
    elif mbl:  # MBL: one head of duration mbl_T, two children of the same tree; spec = <H> / W
        en, H, Ls, K = O.mbl_operators(Nc, prm["mbl_prm_W"], prm["mbl_prm_U"], prm["mbl_prm_J"], int(prm["mbl_seed"]),
                                       int(prm["mbl_mns"]), int(prm["diss_type"]), prm["diss_phase"],
                                       prm["diss_gamma"])
        T = prm["mbl_T"]
        Ut = O.split_tree(K, T, deep)
        U = np.stack([Ut, Ut])
        HE = H
        Rs = np.concatenate([H[None], R]) if nr else H[None]
        ens = O.Ensemble(U, Ls, [1.0] * Ls.shape[0], HE, Rs, T, n, seed=seed, record=int(prm["jump"]), rec_cap=100000)
    else:
        H, Hd, L, K0, K1 = O.dimer_operators(N, prm["dimer_prm_J"], prm["dimer_prm_U"], prm["dimer_prm_E"],
                                             prm["dimer_drv_ampl"], prm["diss_gamma"])
        T = TWO_PI / prm["dimer_drv_freq"]
        t_head = 0.5 * T / nsub if deep_task else T  # init_split_structure_dimer_deep's branch dt
        U = np.stack([O.split_tree(K0, t_head, deep), O.split_tree(K1, t_head, deep)])
        HE = H + prm["dimer_prm_E"] * Hd
        ens = O.Ensemble(U, L, [1.0], HE, R if nr else None, t_head, n, seed=seed, record=int(prm["jump"]),
                         rec_cap=100000)
    ens.init(int(prm["start_type"]), int(prm["start_state"]))
    prop = cfg.get("prop_id", 0)
    period = [0]  # the RK propagator's period_id, reset with the times after the transient

    def advance(k, is_obs=1):
        if deep_task:
            return sum(ens.run_branch_units(b, 2 * nsub, is_obs=is_obs) for _ in range(k) for b in range(2))
        if prop == 0:
            return ens.run_periods(k, is_obs=is_obs)
        Heff = O.dimer_heff(N, prm["dimer_prm_J"], prm["dimer_prm_U"], prm["dimer_prm_E"], prm["diss_gamma"])
        rc = ens.run_periods_rk(k, Heff, Hd, prm["dimer_prm_E"], prm["dimer_drv_ampl"], cfg.get("rk_ns", 1000),
                                period0=period[0], drv_type=int(prm.get("dimer_drv_type", 0)),
                                freq=prm["dimer_drv_freq"], phase=prm.get("dimer_drv_phase", 0.0), is_obs=is_obs)
        period[0] += k
        return rc

    files = {}
    if mbl:  # newdel.cpp:903-905: written to the working directory
        files["energies" + sfx] = f_double_data(en)
    if integ and cfg.get("is_debug", 0):
        files[path + "hamiltonian" + sfx] = f_complex_data(H.reshape(-1))
        for c in range(Ls.shape[0]):
            files[path + "dissipator_%d" % c + sfx] = f_complex_data(Ls[c].reshape(-1))
        files[path + "hamiltonians_qj_0" + sfx] = f_complex_data(K.reshape(-1))
        files[path + "spec_mtx" + sfx] = f_complex_data(S.reshape(-1))
        files[path + "exp_mtx_0" + sfx] = f_complex_data(Ut[-1].reshape(-1))
    elif mbl and cfg.get("is_debug", 0):
        files[path + "hamiltonian" + sfx] = f_complex_data(H.reshape(-1))
        for c in range(Ls.shape[0]):
            files[path + "dissipator_%d" % c + sfx] = f_complex_data(Ls[c].reshape(-1))
        files[path + "hamiltonians_qj_0" + sfx] = f_complex_data(K.reshape(-1))
        files[path + "spec_mtx" + sfx] = f_complex_data(H.reshape(-1))
        files[path + "exp_mtx_0" + sfx] = f_complex_data(Ut[-1].reshape(-1))
    elif cfg.get("is_debug", 0):
        files[path + "hamiltonian" + sfx] = f_complex_data(H.reshape(-1))
        for c, Lc in enumerate(L.reshape(-1, d, d)):
            files[path + "dissipator_%d" % c + sfx] = f_complex_data(Lc.reshape(-1))
        files[path + "hamiltonians_qj_0" + sfx] = f_complex_data(K0.reshape(-1))
        files[path + "hamiltonians_qj_1" + sfx] = f_complex_data(K1.reshape(-1))
        if cfg.get("prop_id", 0) == 0:  # JCS / PS: part 1's tree is engine branch 2
            files[path + "exp_mtx_0" + sfx] = f_complex_data(U[0, -1].reshape(-1))
            files[path + "exp_mtx_1" + sfx] = f_complex_data(U[2 if (jcs or ps) else 1, -1].reshape(-1))
        if jcs:  # JCSDebugBehaviour::save (debugger.cpp:13-26): special = a
            files[path + "spec_mtx" + sfx] = f_complex_data(L.reshape(-1))
        if ps:  # PSDebugBehaviour::save (debugger.cpp:28-53)
            for o, name in enumerate(("spec_mtx", "spec_2_mtx", "spec_3_mtx", "spec_4_mtx")):
                files[path + name + sfx] = f_complex_data(S4[o].reshape(-1))
    if deep_task:
        dp = [0] + [p for p in range(cfg.get("num_obs_periods", 10)) for _ in range(2 * nsub)]
    else:
        dp = O.dump_periods(int(prm["dump_type"]), int(prm["dump_num"]), cfg.get("num_obs_periods", 10))
    ndt = len(dp)
    assert advance(cfg.get("num_tp_periods", 0), is_obs=0) == 0
    ens.t[:] = 0.0
    period[0] = 0
    obs = [ens.observables(is_start=True, want_adr=True)]
    evo_sep, adr_sep = int(prm["dump_evo_sep"]), int(prm["dump_adr_sep"])
    evo_avg, adr_avg_on = int(prm["dump_evo_avg"]), int(prm["dump_adr_avg"])
    phi_evo_on, phi_on = int(prm["dump_phi_evo"]), int(prm["dump_phi"])
    if deep_task:  # StdDeep writes no phi files (experiment.cpp:806-845)
        phi_evo_on = phi_on = 0
    lim = int(prm["jumps_counts"])
    dump_purity = int(prm.get("dump_purity", 0))  # optional key of the drop-in (not in QJX)
    purity = [O.purity(ens.phi)[0]] if dump_purity == 1 else []

    def adr_avg(adr):
        avg = np.zeros(d)
        for tr in range(n):
            avg += adr[tr] / float(n)
        return avg

    acc = {}

    def emit(name, text, append):
        key = path + name
        acc[key] = (acc.get(key, "") if append else "") + text

    if evo_sep == 1 and adr_sep == 1:
        for tr in range(n):
            emit("adr_%d" % tr + sfx, f_double_data(obs[0]["adr"][tr]), False)
    if evo_avg == 1 and adr_avg_on == 1:
        emit("adr_avg" + sfx, f_double_data(adr_avg(obs[0]["adr"])), False)
    if phi_evo_on == 1:
        for tr in range(n):
            emit("phi_evo_%d" % tr + sfx, f_complex_data(ens.phi[tr]), False)
    finished = False
    if deep_task:  # StdDeep obser_process: observables after every sub-period
        for _ in range(cfg.get("num_obs_periods", 10)):
            for b in range(2):
                for _ in range(nsub):
                    assert ens.run_branch_units(b, 2) == 0
                    obs.append(ens.observables(want_adr=True))
                    if evo_sep == 1 and adr_sep == 1:
                        for tr in range(n):
                            emit("adr_%d" % tr + sfx, f_double_data(obs[-1]["adr"][tr]), True)
            if evo_avg == 1 and adr_avg_on == 1:
                emit("adr_avg" + sfx, f_double_data(adr_avg(obs[-1]["adr"])), True)
    for dump_id in range(1, ndt if not deep_task else 1):
        span = dp[dump_id] - dp[dump_id - 1]
        if lim > 0:
            for _ in range(span):
                assert advance(1) == 0
                if np.all(ens.jumps_counts >= lim):
                    finished = True
                    break
        elif span > 0:
            assert advance(span) == 0
        obs.append(ens.observables(want_adr=True))
        if dump_purity == 1:
            purity.append(O.purity(ens.phi)[0])
        if evo_sep == 1 and adr_sep == 1:
            for tr in range(n):
                emit("adr_%d" % tr + sfx, f_double_data(obs[-1]["adr"][tr]), True)
        if phi_evo_on == 1:
            for tr in range(n):
                emit("phi_evo_%d" % tr + sfx, f_complex_data(ens.phi[tr]), True)
        if evo_avg == 1 and adr_avg_on == 1:
            emit("adr_avg" + sfx, f_double_data(adr_avg(obs[-1]["adr"])), True)
        if finished:
            break
    last = obs[-1]
    if dump_purity == 1:
        emit("purity_evo" + sfx, f_double_data(purity), False)
    if jcs or mbl or integ:
        div = alpha if jcs else prm["mbl_prm_W"] if mbl else 1.0
        for o in obs:
            z = o["random_obs"][:, 0]  # result.real /= div; result.imag /= div (real divisions)
            o["spec"] = z.real / div + 1j * (z.imag / div)
            o["random_obs"] = o["random_obs"][:, 1:]
            if mbl:
                o["imbalance"] = O.mbl_imbalance(Nc, o["adr"])
    if mbl and int(prm["dump_obs"]) == 1:
        emit("norm" + sfx, f_double_data(last["norm"]), False)
        emit("spec" + sfx, f_complex_data(last["spec"]), False)
        emit("imbalance" + sfx, f_double_data(last["imbalance"]), False)
    if ps:  # get_spec_ps (/ alpha), get_spec_2_ps, get_spec_3_ps, get_num_photons_ps (experiment.cpp:1568-1708, 2170)
        for o in obs:
            z = o["random_obs"]
            o["spec"] = z[:, 0].real / alpha + 1j * (z[:, 0].imag / alpha)
            o["spec_2"], o["spec_3"], o["mean"] = z[:, 1], z[:, 2], z[:, 3].real.copy()
            o["random_obs"] = z[:, 4:]
    if ps and int(prm["dump_obs"]) == 1:  # PSCoreBehaviour::dump_std (core.cpp:3958-3995)
        emit("norm" + sfx, f_double_data(last["norm"]), False)
        emit("spec" + sfx, f_complex_data(last["spec"]), False)
        emit("spec_2" + sfx, f_complex_data(last["spec_2"]), False)
        emit("spec_3" + sfx, f_complex_data(last["spec_3"]), False)
        emit("mean" + sfx, f_double_data(last["mean"]), False)
    if (jcs or integ) and int(prm["dump_obs"]) == 1:
        emit("norm" + sfx, f_double_data(last["norm"]), False)
        emit("spec" + sfx, f_complex_data(last["spec"]), False)
    if not jcs and not mbl and not integ and not ps and int(prm["dump_obs"]) == 1:
        emit("norm" + sfx, f_double_data(last["norm"]), False)
        emit("mean_start" + sfx, f_double_data(ens.mean_start), False)
        emit("mean" + sfx, f_double_data(last["mean"]), False)
        emit("dispersion" + sfx, f_double_data(last["dispersion"]), False)
        emit("m2" + sfx, f_double_data(last["m2"]), False)
        emit("energy" + sfx, f_double_data(last["energy"]), False)
    if phi_on == 1:
        for tr in range(n):
            emit("phi_%d" % tr + sfx, f_complex_data(ens.phi[tr]), False)
    if phi_evo_on == 1:
        for tr in range(n):
            emit("phi_evo_%d" % tr + sfx, f_complex_data(ens.phi[tr]), True)
    if evo_sep == 1 and int(prm["dump_obs"]) == 1:
        emit("periods" + sfx, f_int_data(dp), False)
        keys = ((("norm", "norm_evo"), ("energy", "mean_evo")) if jcs else
                (("norm", "norm_evo"), ("imbalance", "imbalance_evo")) if mbl else
                (("norm", "norm_evo"),) if integ else
                (("norm", "norm_evo"), ("mean", "mean_evo")) if ps else
                (("norm", "norm_evo"), ("mean", "mean_evo"), ("dispersion", "dispersion_evo"), ("m2", "m2_evo"),
                 ("energy", "energy_evo")))
        for key, name in keys:
            grid = np.zeros((ndt, n))
            for i, o in enumerate(obs):
                grid[i] = o[key]
            emit(name + sfx, f_2d_inv(grid), False)
        if jcs or mbl or integ or ps:
            for key in (("spec", "spec_2", "spec_3") if ps else ("spec",)):
                emit(key + "_evo" + sfx, f_2d_inv_complex(np.array([o[key] for o in obs])), False)
        for o_id in range(nr):
            rows = [o["random_obs"][:, o_id] for o in obs]
            emit("random_obs_evo_%d" % (int(prm["random_obs_seed"]) + o_id) + sfx, f_2d_complex(rows), False)
        if int(prm["jump"]) > 0:
            for tr in range(n):
                t, ty, nm, et = ens.jumps(tr)
                emit("jump_times_%d" % tr + sfx, f_double_data(t), False)
                emit("diss_types_%d" % tr + sfx, f_int_data(ty), False)
                if int(prm["jump"]) > 1:
                    emit("jump_norms_%d" % tr + sfx, f_double_data(nm), False)
                    emit("jump_etas_%d" % tr + sfx, f_double_data(et), False)
    if evo_avg == 0 and adr_avg_on == 1:
        emit("adr_avg" + sfx, f_double_data(adr_avg(last["adr"])), False)
    files.update(acc)
    return files


def expected_lpn_outputs(cfg, prm, R=None):
    """LpnMult (task_id 7): LpnMultExperimentBehaviour::trans_process / obser_process
    (experiment.cpp:138-286) with dump_std, dump_lpn, dump_std_evo, dump_lpn_evo (core.cpp:918-1127)
    and the adr files (dump.cpp:3-98)."""
    sfx_prm, prm = prm, dimersync_as_dimer(cfg, prm)
    nsub = int(prm["deep_num_steps"]) if cfg.get("task_id", 7) == 8 else 0  # LpnMultDeep
    nss = 2 * nsub
    mbl = cfg.get("sys_id", 0) == 3  # MBL: H in observable slot 0, imbalances, MBL file set
    jcs = cfg.get("sys_id", 0) == 1  # JCS: a in observable slot 0, <a^+ a>, JCS file set
    integ = cfg.get("sys_id", 0) in (5, 7, 8, 9)  # Integrable, Floquet: the special matrix in slot 0
    spec = mbl or jcs or integ
    N = 0 if (mbl or integ) else int(prm["N"])
    d = N if jcs else N + 1
    if mbl:
        Nc, W = int(prm["mbl_Nc"]), float(prm["mbl_prm_W"])
        d = len(O.mbl_basis(Nc))
    if jcs:
        W = float(prm["jcs_prm_alpha"])  # the spec divisor
    if integ:
        d = {7: 4, 8: 1 << int(prm.get("flqnsp_n", 0)), 9: 2 * (int(prm.get("flq_sp_ph_n_ph", 0)) + 1)}.get(
            cfg.get("sys_id", 0), 1 << int(prm.get("integrable_N", 0)))
        W = 1.0
    n = cfg["num_trajectories"]
    half = n // 2
    deep = cfg.get("ex_deep", 16)
    seed = cfg.get("seed", 0)
    path = cfg.get("path", "")
    sfx = suffix(cfg, sfx_prm)
    nr = int(prm["num_random_obs"])
    if jcs:
        alpha = W
        H, Hd, L, Nop, K0, K1 = O.jcs_operators(N, alpha, prm["jcs_drv_ampl"])
        heads = [prm["jcs_drv_part_1"] * alpha, prm["jcs_drv_part_2"] * alpha]
        U0, U1 = O.split_tree(K0, heads[0], deep), O.split_tree(K1, heads[1], deep)
        U = np.stack([U0, U0, U1, U1])
        Rs = np.concatenate([L[None], R]) if nr else L[None]
        T = alpha
        calc_T = heads[0] + heads[1]  # JCSCoreBehaviour::calc_T (core.cpp:2833-2845)
        ens = O.Ensemble(U, L, [1.0], Nop, Rs, T, n, seed=seed, record=int(prm["jump"]), rec_cap=100000,
                         branch_len=[0.5 * heads[0], 0.5 * heads[0], 0.5 * heads[1], 0.5 * heads[1]])
    elif integ:
        L, S, H, T, U, _ = spec_system(cfg, prm, deep)
        calc_T = T
        Rs = np.concatenate([S[None], R]) if nr else S[None]
        ens = O.Ensemble(U, L, [1.0] * L.shape[0], H, Rs, T, n, seed=seed, record=int(prm["jump"]), rec_cap=100000)
    elif mbl:
        en, H, L, K = O.mbl_operators(Nc, W, prm["mbl_prm_U"], prm["mbl_prm_J"], int(prm["mbl_seed"]),
                                      int(prm["mbl_mns"]), int(prm["diss_type"]), prm["diss_phase"], prm["diss_gamma"])
        T = prm["mbl_T"]
        Ut = O.split_tree(K, T, deep)
        Rs = np.concatenate([H[None], R]) if nr else H[None]
        ens = O.Ensemble(np.stack([Ut, Ut]), L, [1.0] * L.shape[0], H, Rs, T, n, seed=seed, record=int(prm["jump"]),
                         rec_cap=100000)
        calc_T = T
    else:
        H, Hd, L, K0, K1 = O.dimer_operators(N, prm["dimer_prm_J"], prm["dimer_prm_U"], prm["dimer_prm_E"],
                                             prm["dimer_drv_ampl"], prm["diss_gamma"])
        T = TWO_PI / prm["dimer_drv_freq"]
        # LpnMultDeep (task_id 8): the split trees of the sub-period T / (2 deep_num_steps)
        t_head = 0.5 * T / nsub if nsub else T
        U = np.stack([O.split_tree(K0, t_head, deep), O.split_tree(K1, t_head, deep)])
        HE = H + prm["dimer_prm_E"] * Hd
        ens = O.Ensemble(U, L, [1.0], HE, R if nr else None, t_head, n, seed=seed, record=int(prm["jump"]),
                         rec_cap=100000)
        calc_T = T
    ens.init(int(prm["start_type"]), int(prm["start_state"]))
    prop = cfg.get("prop_id", 0)
    period = [0]

    def advance(k, is_obs=1, tr1=None):
        if nsub:  # deep: a period is 2 deep_num_steps units of each branch
            return sum(ens.run_branch_units(b, nss, is_obs=is_obs, tr1=tr1) for _ in range(k) for b in range(2))
        if prop == 0:
            return ens.run_periods(k, is_obs=is_obs, tr1=tr1)
        Heff = O.dimer_heff(N, prm["dimer_prm_J"], prm["dimer_prm_U"], prm["dimer_prm_E"], prm["diss_gamma"])
        rc = ens.run_periods_rk(k, Heff, Hd, prm["dimer_prm_E"], prm["dimer_drv_ampl"], cfg.get("rk_ns", 1000),
                                period0=period[0], drv_type=int(prm.get("dimer_drv_type", 0)),
                                freq=prm["dimer_drv_freq"], phase=prm.get("dimer_drv_phase", 0.0), is_obs=is_obs,
                                tr1=tr1)
        period[0] += k
        return rc

    max_energy = float(np.max(np.abs(np.diag(H).real))) if not integ else 0.0
    lp = O.Lpn(ens, lpn_type=int(prm["lpn_type"]), eps_deep=int(prm["lpn_eps_deep"]),
               eps_low=float(prm["lpn_eps_low"]), eps_high=float(prm["lpn_eps_high"]),
               eps_error=float(prm["lpn_eps_error"]), delta_s=float(prm["lpn_delta_s"]),
               delta_f_high=float(prm["lpn_delta_f_high"]), delta_f_low=float(prm["lpn_delta_f_low"]),
               per_period=int(prm["lambda_per_periods"]) != 0, max_energy=max_energy,
               mbl_Nc=Nc if mbl else 0, spec_div=W if spec else 1.0,
               chars_sys={6: 0, 7: 5, 8: 5, 9: 5}.get(cfg.get("sys_id", 0), cfg.get("sys_id", 0)))  # DimerSync, Floq*
    if nsub:  # init_dump_periods_deep (newdel_exp.cpp:377-406)
        dp = [0] + [p for p in range(cfg.get("num_obs_periods", 10)) for _ in range(nss)]
    else:
        dp = O.dump_periods(int(prm["dump_type"]), int(prm["dump_num"]), cfg.get("num_obs_periods", 10))
    ndt = len(dp)
    assert advance(cfg.get("num_tp_periods", 0), is_obs=0, tr1=half) == 0
    lp.start()
    ens.t[:] = 0.0
    period[0] = 0
    obs = [ens.observables(is_start=True, want_adr=True)]
    if mbl:
        obs[0]["imbalance"] = O.mbl_imbalance(Nc, obs[0]["adr"])
    lpn = [lp.values()]
    save_lambdas = int(prm["save_lambdas"])
    recs = {k: [[] for _ in range(n)] for k in ("ratio", "delta_s", "delta_f")}
    evo_sep, adr_sep = int(prm["dump_evo_sep"]), int(prm["dump_adr_sep"])
    evo_avg, adr_avg_on = int(prm["dump_evo_avg"]), int(prm["dump_adr_avg"])
    acc = {}

    def emit(name, text, append):
        key = path + name
        acc[key] = (acc.get(key, "") if append else "") + text

    def adr_avg(adr, m):
        avg = np.zeros(d)
        for tr in range(m):
            avg += adr[tr] / float(m)
        return avg

    if evo_sep == 1 and adr_sep == 1:
        for tr in range(n):
            emit("adr_%d" % tr + sfx, f_double_data(obs[0]["adr"][tr]), False)
    if evo_avg == 1 and adr_avg_on == 1:
        emit("adr_avg" + sfx, f_double_data(adr_avg(obs[0]["adr"], n)), False)
    if nsub and int(prm["dump_phi_evo"]) == 1:
        for tr in range(n):
            emit("phi_evo_%d" % tr + sfx, f_complex_data(ens.phi[tr]), False)
    for p in range(cfg.get("num_obs_periods", 10) if nsub else 0):  # ex_period_obs_deep_mult_lpn
        for b in range(2):
            for k in range(nsub):
                dump_id = p * nss + b * nsub + k + 1
                assert ens.run_branch_units(b, 2) == 0
                o = ens.observables(want_adr=True)
                if lp.cfg.per_period == 0 or (b == 1 and k == nsub - 1):
                    lp.period(float(dump_id) / float(nss) * calc_T)
                    o["adr"][half:] = ens.observables(want_adr=True)["adr"][half:]
                    last = lp.last()
                    for v in range(half, n):
                        if save_lambdas > 0 and last["renormed"][v]:
                            for kk in recs:
                                recs[kk][v].append(last[kk][v])
                else:
                    lp.bases()
                obs.append(o)
                lpn.append(lp.values())
                if evo_sep == 1 and adr_sep == 1:
                    for tr in range(n):
                        emit("adr_%d" % tr + sfx, f_double_data(o["adr"][tr]), True)
        if evo_avg == 1 and adr_avg_on == 1:
            emit("adr_avg" + sfx, f_double_data(adr_avg(obs[-1]["adr"], half)), True)
    for dump_id in range(1, ndt if not nsub else 1):
        o = {k: v.copy() for k, v in obs[-1].items()}
        for period_id in range(dp[dump_id - 1], dp[dump_id]):
            assert advance(1) == 0
            o = ens.observables(want_adr=True)
            if mbl:  # calc_chars_std before lambda_lpn: the pre-update adr rows
                o["imbalance"] = O.mbl_imbalance(Nc, o["adr"])
            lp.period((period_id + 1) * calc_T)
            if not jcs:  # JCS's calc_chars_lpn does not rewrite abs_diag_rho_all
                o["adr"][half:] = ens.observables(want_adr=True)["adr"][half:]
            last = lp.last()
            for v in range(half, n):
                if save_lambdas > 0 and last["renormed"][v]:
                    for k in recs:
                        recs[k][v].append(last[k][v])
        obs.append(o)
        lpn.append(lp.values())
        if evo_sep == 1 and adr_sep == 1:
            for tr in range(n):
                emit("adr_%d" % tr + sfx, f_double_data(o["adr"][tr]), True)
        if evo_avg == 1 and adr_avg_on == 1:
            emit("adr_avg" + sfx, f_double_data(adr_avg(o["adr"], half)), True)
    last = obs[-1]
    ro = 1 if spec else 0
    if spec:
        for o in obs:
            z = o["random_obs"][:, 0]
            o["spec"] = z.real / W + 1j * (z.imag / W)
        for v in lpn:
            z = v["robs_lpn"][:, 0]
            v["spec_lpn"] = z.real / W + 1j * (z.imag / W)
    if mbl and int(prm["dump_obs"]) == 1:
        emit("norm" + sfx, f_double_data(last["norm"]), False)
        emit("spec" + sfx, f_complex_data(last["spec"]), False)
        emit("imbalance" + sfx, f_double_data(last["imbalance"]), False)
        emit("lambda" + sfx, f_double_data(lpn[-1]["lambda_now"]), False)
        emit("num_renorms" + sfx, f_int_data(lpn[-1]["num_renorms"]), False)
        emit("spec_lpn" + sfx, f_complex_data(lpn[-1]["spec_lpn"]), False)
        emit("imbalance_lpn" + sfx, f_double_data(lpn[-1]["mean_lpn"]), False)
    if integ and int(prm["dump_obs"]) == 1:
        emit("norm" + sfx, f_double_data(last["norm"]), False)
        emit("spec" + sfx, f_complex_data(last["spec"]), False)
        emit("lambda" + sfx, f_double_data(lpn[-1]["lambda_now"]), False)
        emit("num_renorms" + sfx, f_int_data(lpn[-1]["num_renorms"]), False)
        emit("spec_lpn" + sfx, f_complex_data(lpn[-1]["spec_lpn"]), False)
    if jcs and int(prm["dump_obs"]) == 1:
        emit("norm" + sfx, f_double_data(last["norm"]), False)
        emit("spec" + sfx, f_complex_data(last["spec"]), False)
        emit("lambda" + sfx, f_double_data(lpn[-1]["lambda_now"]), False)
        emit("num_renorms" + sfx, f_int_data(lpn[-1]["num_renorms"]), False)
        emit("spec_lpn" + sfx, f_complex_data(lpn[-1]["spec_lpn"]), False)
        emit("mean" + sfx, f_double_data(lpn[-1]["mean_lpn"]), False)
    if int(prm["dump_obs"]) == 1 and not spec:
        emit("norm" + sfx, f_double_data(last["norm"]), False)
        emit("mean_start" + sfx, f_double_data(ens.mean_start), False)
        emit("mean" + sfx, f_double_data(last["mean"]), False)
        emit("dispersion" + sfx, f_double_data(last["dispersion"]), False)
        emit("m2" + sfx, f_double_data(last["m2"]), False)
        emit("energy" + sfx, f_double_data(last["energy"]), False)
        emit("lambda" + sfx, f_double_data(lpn[-1]["lambda_now"]), False)
        emit("num_renorms" + sfx, f_int_data(lpn[-1]["num_renorms"]), False)
        emit("mean_lpn" + sfx, f_double_data(lpn[-1]["mean_lpn"]), False)
        emit("energy_lpn" + sfx, f_double_data(lpn[-1]["energy_lpn"]), False)
    if int(prm["dump_obs"]) == 1:
        if save_lambdas > 0:
            for tr in range(n):
                emit("delta_f_by_delta_s_%d" % tr + sfx, f_double_data(recs["ratio"][tr]), False)
                emit("deltas_s_%d" % tr + sfx, f_double_data(recs["delta_s"][tr]), False)
                emit("deltas_f_%d" % tr + sfx, f_double_data(recs["delta_f"][tr]), False)
    if evo_sep == 1 and int(prm["dump_obs"]) == 1:
        emit("periods" + sfx, f_int_data(dp), False)
        keys = ((("norm", "norm_evo"), ("imbalance", "imbalance_evo")) if mbl else
                (("norm", "norm_evo"), ("energy", "mean_evo")) if jcs else
                (("norm", "norm_evo"),) if integ else
                (("norm", "norm_evo"), ("mean", "mean_evo"), ("dispersion", "dispersion_evo"), ("m2", "m2_evo"),
                 ("energy", "energy_evo")))
        for key, name in keys:
            emit(name + sfx, f_2d_inv(np.array([o[key] for o in obs])), False)
        if spec:
            emit("spec_evo" + sfx, f_2d_inv_complex(np.array([o["spec"] for o in obs])), False)
        for o_id in range(nr):
            rows = [o["random_obs"][:, ro + o_id] for o in obs]
            emit("random_obs_evo_%d" % (int(prm["random_obs_seed"]) + o_id) + sfx, f_2d_complex(rows), False)
        if int(prm["jump"]) > 0:
            for tr in range(n):
                t, ty, nm, et = ens.jumps(tr)
                emit("jump_times_%d" % tr + sfx, f_double_data(t), False)
                emit("diss_types_%d" % tr + sfx, f_int_data(ty), False)
                if int(prm["jump"]) > 1:
                    emit("jump_norms_%d" % tr + sfx, f_double_data(nm), False)
                    emit("jump_etas_%d" % tr + sfx, f_double_data(et), False)
        keys = ((("lambda_now", "lambda_evo"), ("mean_lpn", "imbalance_lpn_evo")) if mbl else
                (("lambda_now", "lambda_evo"), ("mean_lpn", "mean_lpn_evo")) if jcs else
                (("lambda_now", "lambda_evo"),) if integ else
                (("lambda_now", "lambda_evo"), ("mean_lpn", "mean_lpn_evo"), ("energy_lpn", "energy_lpn_evo")))
        for key, name in keys:
            emit(name + sfx, f_2d_inv(np.array([v[key] for v in lpn])), False)
        if spec:
            emit("spec_lpn_evo" + sfx, f_2d_inv_complex(np.array([v["spec_lpn"] for v in lpn])), False)
        for o_id in range(nr):
            rows = [v["robs_lpn"][:, ro + o_id] for v in lpn]
            emit("random_obs_lpn_evo_%d" % (int(prm["random_obs_seed"]) + o_id) + sfx, f_2d_complex(rows), False)
    if evo_avg == 0 and adr_avg_on == 1:
        emit("adr_avg" + sfx, f_double_data(adr_avg(last["adr"], half)), False)
    if mbl:  # newdel.cpp:903-905: written to the working directory
        acc["energies" + sfx] = f_double_data(en)
    return acc


JCS_PARAMS = {"N": 40, "jcs_prm_alpha": 5.0, "jcs_drv_ampl": 3.2, "jcs_drv_part_1": 0.5, "jcs_drv_part_2": 1.5}

# a Floquet two-spin system (its QJ branch is undriven: flq2sp_ampl enters the RK propagator only)
FLOQ2_PARAMS = {"flq2sp_ampl": 1.0, "flq2sp_freq": 1.0, "flq2sp_Delta_1": 1.0, "flq2sp_Delta_2": 0.6, "flq2sp_J": 0.4,
                "flq2sp_gamma": 0.3}

# a Floquet many-spin system (3 spins; sy (x) sy (x) sy is imaginary)
FLOQN_PARAMS = {"flqnsp_n": 3, "flqnsp_ampl": 1.0, "flqnsp_freq": 1.0, "flqnsp_Delta": 1.0, "flqnsp_J": 0.4,
                "flqnsp_gamma": 0.3}

# a Floquet spin-photon system (up to 8 photons, d = 18).  Its state |0 photons, spin 1> is dark (no loss,
# isolated), where repeated matvecs let the norm drift an ulp above 1, which the reference rejects
# ("norm more than 1", experiment.cpp:1247-1251): the test starts high in the photon ladder with weak loss
FLOQP_PARAMS = {"flq_sp_ph_n_ph": 8, "flq_sp_ph_ampl": 1.0, "flq_sp_ph_freq": 1.0, "flq_sp_ph_Delta": 1.0,
                "flq_sp_ph_Omega": 0.5, "flq_sp_ph_gamma": 0.02}

# a DimerSync system (two drives; the QJ branches carry drive 1, the period is drive 2's)
DIMERSYNC_PARAMS = {"dimersync_N": 16, "dimersync_prm_E": 1.0, "dimersync_prm_U": 0.5, "dimersync_prm_J": 1.0,
                    "dimersync_drv_ampl_1": 1.5, "dimersync_drv_freq_1": 1.0, "dimersync_drv_phase_1": 0.0,
                    "dimersync_drv_ampl_2": 0.5, "dimersync_drv_freq_2": 2.0, "dimersync_drv_phase_2": 0.25,
                    "dimersync_main_period": 2}

# submit_ps.py's system (1 spin, alpha 5, parts 1 / 1 (x T), diss_w 0.05; 300 photon states there, 24 here)
PS_PARAMS = {"ps_num_spins": 1, "ps_num_photons_states": 24, "ps_prm_alpha": 5.0, "ps_prm_d": 1.0, "ps_prm_g": 0.5,
             "ps_drv_ampl": 3.2, "ps_drv_part_1": 0.5, "ps_drv_part_2": 1.5, "ps_diss_w": 0.05, "diss_type": 1}

# submit_integrable.py's system (tau 1, k -1, integrable_N 7 there; 6 spins here), one disorder seed
INTEGRABLE_PARAMS = {"integrable_N": 6, "integrable_seed": 2, "integrable_num_seeds": 1000000, "integrable_tau": 1.0,
                     "integrable_k": -1.0, "integrable_T": 1.0}

# the production MBL sweeps' values (Nc 8, diss_type 1, gamma 0.1, J 1, T 10), one disorder seed
MBL_PARAMS = {"mbl_Nc": 8, "mbl_seed": 3, "mbl_mns": 1000000, "mbl_prm_W": 2.5, "mbl_prm_U": 1.0, "mbl_prm_J": 1.0,
              "mbl_T": 10.0, "diss_type": 1, "diss_gamma": 0.1, "diss_phase": 0.0}

LPN_PARAMS = {
    "lpn_type": 0, "lpn_eps_deep": 100, "lpn_eps_error": 1.0e-10, "lpn_eps_high": 10, "lpn_eps_low": -10,
    "lpn_delta_s": 1.0e-3, "lpn_delta_f_high": 1.0e-1, "lpn_delta_f_low": 1.0e-5, "lambda_per_periods": 0,
    "save_lambdas": 0,
}

BASE_PARAMS = {
    "num_random_obs": 1, "random_obs_seed": 100, "random_obs_mns": 1000000, "random_obs_type": 2,
    "dump_obs": 1, "dump_phi": 0, "dump_phi_evo": 0, "dump_adr_sep": 0, "dump_adr_avg": 0, "dump_evo_sep": 1,
    "dump_evo_avg": 0, "dump_type": 0, "dump_num": 3, "N": 16, "diss_type": 0, "diss_gamma": 0.1,
    "diss_phase": 0.0, "dimer_drv_type": 0, "dimer_drv_ampl": 1.5, "dimer_drv_freq": 1.0, "dimer_drv_phase": 0.0,
    "dimer_prm_E": 1.0, "dimer_prm_U": 0.5, "dimer_prm_J": 1.0, "start_type": 0, "start_state": 0,
    "jump": 2, "jumps_counts": 0,
}

BASE_CONFIG = {
    "sys_id": 0, "task_id": 1, "prop_id": 0, "is_debug": 0, "is_pp": 0, "seed": 3, "mns": 1000000,
    "num_threads": 4, "num_trajectories": 12, "num_tp_periods": 2, "num_obs_periods": 6, "ex_deep": 16, "rk_ns": 100,
}
