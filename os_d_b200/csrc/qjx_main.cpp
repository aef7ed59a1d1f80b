// qjx_main.cpp -- qjx_b200: process-level drop-in for the reference's qjx executable on the
// Std task (task_id 1) and the LpnMult task (task_id 7) with the QJ propagator (prop_id 0) or the
// RK propagator (prop_id 1), and the StdDeep task (task_id 4, QJ propagator), for the dimer (sys_id 0);
// the Std and LpnMult tasks with the QJ propagator for the JCS (sys_id 1), MBL (sys_id 3) and
// Integrable (sys_id 5) systems, the Std task with the QJ propagator for PS (sys_id 2), and the
// Std and LpnMult tasks with the QJ propagator for DimerSync (sys_id 6, whose QJ branches are the
// dimer's with its first drive; the second drive enters the RK propagator only), and Floq2Spins
// FloqManySpins and FloqSpinPh (sys_id 7, 8, 9: Std and LpnMult with their undriven QJ branches).
//
// Flow of the generic main + Processor::process (source/cpp/QJX/QJX/main.cpp:3-192,
// processor.cpp:50-76): read ./config.txt and ./params.txt, build the dimer model, run the
// transient periods, take dump 0 (calc_chars_std_start), run the observation periods with
// observables at every dump, and write the reference's files (core.cpp:918-1084,
// dump.cpp:3-61, core.cpp:12567-12613) under `path` with the same names and formats.
// The trajectories run on the GPU through the C ABI of libqjx_b200.so.
//
//   qjx_b200 [--config FILE] [--params FILE] [--device N] [--check]
// --check parses both files, prints the parameter echo and the file-name suffix, and exits
// without touching a GPU.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qjx_b200.h"
#include "qjx_config.h"

using namespace qjxio;

namespace {

[[noreturn]] void die(const std::string &msg)
{
    std::cout << "Error: " << msg << std::endl;
    std::exit(EXIT_FAILURE);
}

void check(qjx_status s, qjx_engine *h, const char *what)
{
    if (s == QJX_OK) return;
    std::string m = std::string(what) + " failed: " + qjx_status_string(s);
    if (h) m += std::string(" (") + qjx_last_error(h) + ")";
    die(m);
}

struct Dumps {
    std::vector<double> norm, mean, disp, m2, energy;  // [dump][tr]
    std::vector<std::complex<double>> robs;           // [dump][tr][nr]
};

void write_2d_inv(const std::string &fn, const std::vector<double> &v, int nrec, int ndt, int n)
{
    std::vector<double> inv((size_t)ndt * n, 0.0);  // [tr][dump] like ed->*_evo
    for (int dmp = 0; dmp < nrec; dmp++)
        for (int tr = 0; tr < n; tr++) inv[(size_t)tr * ndt + dmp] = v[(size_t)dmp * n + tr];
    save_2d_inv_double_data(fn, inv.data(), ndt, n, 16, false);
}

// LpnMult (task_id 7): LpnMultExperimentBehaviour::trans_process / obser_process
// (experiment.cpp:138-286).  The bases [0, n/2) run the transient alone, every variation
// n/2 + b starts as its base perturbed to delta_s, and after every observation period the
// variations' Lyapunov sums are updated (lambda_lpn / lambda_lpn_now).  Files: dump_std,
// dump_lpn, dump_std_evo, dump_lpn_evo (core.cpp:918-1127), adr files (dump.cpp:3-98).
// JCS (sys_id 1; JCSCoreBehaviour, core.cpp:2739-3150) and MBL (sys_id 3; MBLCoreBehaviour,
// core.cpp:4677-5105): the spec operator (a or H) rides in random-observable slot 0, spec = slot 0
// / spec_div (alpha or W); the mean characteristics are <a^+ a> (JCS) or imbalances (MBL); each
// system writes its own file set.  calc_T is the period of the Lyapunov time (calc_T: JCS
// part_1 alpha + part_2 alpha, core.cpp:2833-2845).
// LpnMultDeep (task_id 8, the dimer; nsub = deep_num_steps > 0): the same pairs advanced one
// sub-period at a time (LpnMultDeepExperimentBehaviour::obser_process, experiment.cpp:302-350;
// ex_period_obs_deep_mult_lpn, core.cpp:155-241): the Lyapunov step after every sub-period at
// curr_time = dump_id / (2 nsub) T (lambda_per_periods 0) or at the last sub-period of each period
// (lambda_per_periods 1; the bases' characteristics only in between), one dump per sub-period.
void run_lpn_mult(qjx_engine *h, const RunParam &rp, const ConfigParam &cp, const qjx_config &cfg,
                  const std::vector<double> &H, int d, int num_robs, int robs_seed, int sys, int Nc, double spec_div,
                  double calc_T, int nsub)
{
    const bool mbl = sys == 3, jcs = sys == 1, integ = sys == 5, spec = mbl || jcs || integ;
    const double W = spec_div;
    const int ro = spec ? 1 : 0, nr = num_robs + ro;  // engine slots: [spec,] random observables
    const int n = cp.num_trajectories, half = n / 2;
    if (n < 2 || (n & 1)) die("LpnMult needs an even num_trajectories >= 2");
    const std::string &sfx = cp.fn_suffix;
    const std::string path = rp.path;
    const int dump_obs = int(param(cp, "dump_obs")), dump_evo_sep = int(param(cp, "dump_evo_sep"));
    const int dump_evo_avg = int(param(cp, "dump_evo_avg")), dump_adr_sep = int(param(cp, "dump_adr_sep"));
    const int dump_adr_avg_on = int(param(cp, "dump_adr_avg"));
    const int jump = int(param(cp, "jump"));
    qjx_lpn_config lc{};
    lc.lpn_type = int(param(cp, "lpn_type"));
    lc.eps_deep = int(param(cp, "lpn_eps_deep"));
    lc.per_period = int(param(cp, "lambda_per_periods")) == 0 ? 0 : 1;
    lc.eps_low = param(cp, "lpn_eps_low");
    lc.eps_high = param(cp, "lpn_eps_high");
    lc.eps_error = param(cp, "lpn_eps_error");
    lc.delta_s = param(cp, "lpn_delta_s");
    lc.delta_f_high = param(cp, "lpn_delta_f_high");
    lc.delta_f_low = param(cp, "lpn_delta_f_low");
    const int save_lambdas = int(param(cp, "save_lambdas"));
    lc.mbl_Nc = mbl ? Nc : 0;
    lc.chars_sys = sys;
    lc.spec_div = spec_div;
    lc.max_energy = 0.0;  // init_obs_lpn (newdel_exp.cpp:540-550)
    for (int st = 0; st < d; st++) {
        const double v = std::fabs(H[2 * ((size_t)st * d + st)]);
        if (v > lc.max_energy) lc.max_energy = v;
    }
    const int nss = 2 * nsub;  // sub-periods per period (num_ham_qj deep_num_steps)
    std::vector<int> dp;
    if (nsub > 0) {  // init_dump_periods_deep (newdel_exp.cpp:377-406)
        dp.push_back(0);
        for (int p = 0; p < cp.num_obs_periods; p++)
            for (int k = 0; k < nss; k++) dp.push_back(p);
    } else {
        dp = dump_periods(int(param(cp, "dump_type")), int(param(cp, "dump_num")), cp.num_obs_periods);
    }
    if (dp.empty()) die("Wrong dump_type");
    const int ndt = (int)dp.size();

    // per-dump records: std observables live in the engine's dump slots; Lyapunov values here
    std::vector<double> lam_evo, mean_lpn_evo, energy_lpn_evo;
    std::vector<std::complex<double>> robs_lpn_evo;
    std::vector<double> lam(n), mean_l(n), energy_l(n);
    std::vector<std::complex<double>> robs_l((size_t)n * (nr ? nr : 1));
    std::vector<int> renorms(n);
    auto take_lpn = [&]() {
        check(qjx_lpn_get(h, lam.data(), nullptr, nullptr, mean_l.data(), energy_l.data(),
                          nr ? reinterpret_cast<double *>(robs_l.data()) : nullptr, renorms.data()),
              h, "qjx_lpn_get");
        lam_evo.insert(lam_evo.end(), lam.begin(), lam.end());
        mean_lpn_evo.insert(mean_lpn_evo.end(), mean_l.begin(), mean_l.end());
        energy_lpn_evo.insert(energy_lpn_evo.end(), energy_l.begin(), energy_l.end());
        robs_lpn_evo.insert(robs_lpn_evo.end(), robs_l.begin(), robs_l.begin() + (size_t)n * nr);
    };
    // MBL: the std imbalance of a dump comes from its adr rows before the Lyapunov update rewrites
    // the variations' rows (calc_chars_std runs before lambda_lpn, experiment.cpp:226-252)
    std::vector<double> imb_std(mbl ? (size_t)ndt * n : 0);
    auto take_imbalance = [&](int dump) {
        if (!mbl) return;
        std::vector<double> adr((size_t)n * d);
        check(qjx_get_observables(h, dump, 1, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, adr.data()), h,
              "qjx_get_observables");
        check(qjx_mbl_imbalance(Nc, n, adr.data(), imb_std.data() + (size_t)dump * n), h, "qjx_mbl_imbalance");
    };
    // save_lambdas: delta_f / delta_s, delta_s, delta_f of every renormalisation per trajectory
    std::vector<std::vector<double>> rec_ratio(n), rec_ds(n), rec_df(n);
    std::vector<int> ren(n), iters(n);
    std::vector<double> ratio(n), rds(n), rdf(n), eps(n);
    auto after_lpn = [&](bool start) {
        if (save_lambdas <= 0 && rp.is_pp != 1) return;
        check(qjx_lpn_get_last(h, ren.data(), ratio.data(), rds.data(), rdf.data(), iters.data(), eps.data()), h,
              "qjx_lpn_get_last");
        std::vector<double> ds_now(n);
        if (rp.is_pp == 1)
            check(qjx_lpn_get(h, nullptr, nullptr, ds_now.data(), nullptr, nullptr, nullptr, nullptr), h, "qjx_lpn_get");
        for (int v = half; v < n; v++) {
            if (!start && !ren[v]) continue;
            if (!start && save_lambdas > 0) {
                rec_ratio[v].push_back(ratio[v]);
                rec_ds[v].push_back(rds[v]);
                rec_df[v].push_back(rdf[v]);
            }
            if (rp.is_pp == 1)  // var_trajectory_lpn's progress lines (experiment.cpp:2385-2392)
                std::cout << "lpn: " << v + 1 << std::endl
                          << "curr_lpn_eps: " << std::log10(eps[v]) << std::endl
                          << "lpn_deep: " << iters[v] << std::endl
                          << "delta_s: " << ds_now[v] << std::endl
                          << std::endl;
        }
    };
    auto get_adr = [&](int dump) {
        std::vector<double> adr((size_t)n * d);
        check(qjx_get_observables(h, cfg.keep_adr ? dump : 0, 1, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                  adr.data()),
              h, "qjx_get_observables");
        return adr;
    };
    auto write_adr_single = [&](int dump, bool append) {
        if (!(dump_evo_sep == 1 && dump_adr_sep == 1)) return;
        const std::vector<double> adr = get_adr(dump);
        for (int tr = 0; tr < n; tr++)
            save_double_data(path + "adr_" + std::to_string(tr) + sfx, adr.data() + (size_t)tr * d, d, 16, append);
    };
    auto write_adr_avg = [&](int dump, int tr1, bool append) {  // dump_adr_avg / dump_adr_avg_mult
        if (dump_adr_avg_on != 1) return;
        const std::vector<double> adr = get_adr(dump);
        std::vector<double> avg(d, 0.0);
        for (int tr = 0; tr < tr1; tr++)
            for (int st = 0; st < d; st++) avg[st] += adr[(size_t)tr * d + st] / double(tr1);
        save_double_data(path + "adr_avg" + sfx, avg.data(), d, 16, append);
    };

    // trans_process: the bases' transient, then copy + perturb, refresh times, dump 0
    check(qjx_init_thresholds(h), h, "qjx_init_thresholds");
    check(qjx_set_active(h, half), h, "qjx_set_active");
    check(qjx_run_periods(h, cp.num_tp_periods, 0, nullptr, 0, 0), h, "qjx_run_periods");
    check(qjx_set_active(h, n), h, "qjx_set_active");
    check(qjx_lpn_start(h, &lc), h, "qjx_lpn_start");
    after_lpn(true);
    check(qjx_reset_times(h), h, "qjx_reset_times");
    check(qjx_observe(h, 0, 1), h, "qjx_observe");
    take_imbalance(0);
    take_lpn();
    write_adr_single(0, false);
    if (dump_evo_avg == 1) write_adr_avg(0, n, false);

    std::vector<bool> zero_span(ndt, false);
    if (nsub > 0) {  // LpnMultDeep obser_process: sub-period by sub-period
        if (int(param(cp, "dump_phi_evo")) == 1) {  // dump_phi_evo(ad, false) (core.cpp:12591-12613)
            std::vector<double> psi(2 * (size_t)n * d);
            check(qjx_get_states(h, psi.data(), nullptr, nullptr, nullptr), h, "qjx_get_states");
            for (int tr = 0; tr < n; tr++)
                save_complex_data(path + "phi_evo_" + std::to_string(tr) + sfx, psi.data() + 2 * (size_t)tr * d, d, 16,
                                  false);
        }
        for (int p = 0; p < cp.num_obs_periods; p++) {
            if (rp.is_pp == 1) std::cout << "dump_id: " << p + 1 << std::endl;
            for (int k = 0; k < nss; k++) {
                const int dump_id = p * nss + k + 1;
                check(qjx_run_sub_periods(h, 1, dump_id), h, "qjx_run_sub_periods");
                if (lc.per_period == 0 || k == nss - 1) {
                    check(qjx_lpn_period(h, double(dump_id) / double(nss) * calc_T, dump_id), h, "qjx_lpn_period");
                    after_lpn(false);
                } else {
                    check(qjx_lpn_bases(h), h, "qjx_lpn_bases");
                }
                take_lpn();
                write_adr_single(dump_id, true);
            }
            if (dump_evo_avg == 1) write_adr_avg((p + 1) * nss, half, true);
        }
    }
    // obser_process: period by period (the Lyapunov update follows every period)
    for (int dump_id = 1; dump_id < ndt && nsub == 0; dump_id++) {
        if (rp.is_pp == 1) std::cout << "dump_id: " << dump_id << std::endl;
        for (int period_id = dp[dump_id - 1]; period_id < dp[dump_id]; period_id++) {
            const bool at_dump = period_id + 1 == dp[dump_id];
            const int one = 1;
            check(qjx_run_periods(h, 1, 1, at_dump ? &one : nullptr, at_dump ? 1 : 0, dump_id), h, "qjx_run_periods");
            if (at_dump) take_imbalance(dump_id);
            // JCS's calc_chars_lpn leaves abs_diag_rho_all alone: its adr rows stay the std ones
            check(qjx_lpn_period(h, double(period_id + 1) * calc_T, (at_dump && !jcs) ? dump_id : -1), h,
                  "qjx_lpn_period");
            after_lpn(false);
        }
        if (dp[dump_id] == dp[dump_id - 1]) {  // no period ran: adr of the current states (abs_diag_rho_all)
            check(qjx_observe(h, dump_id, 0), h, "qjx_observe");
            zero_span[dump_id] = true;
        }
        take_lpn();
        write_adr_single(dump_id, true);
        if (dump_evo_avg == 1) write_adr_avg(dump_id, half, true);
    }
    const int last_dump = ndt - 1;

    std::vector<double> norm_((size_t)ndt * n), mean_((size_t)ndt * n), disp_((size_t)ndt * n), m2_((size_t)ndt * n),
        energy_((size_t)ndt * n);
    std::vector<std::complex<double>> robs_((size_t)ndt * n * (nr ? nr : 1));
    check(qjx_get_observables(h, 0, ndt, norm_.data(), mean_.data(), disp_.data(), m2_.data(), energy_.data(),
                              nr ? reinterpret_cast<double *>(robs_.data()) : nullptr, nullptr),
          h, "qjx_get_observables");
    // a dump with no period since the previous one repeats the previous std characteristics
    // (calc_chars_std runs once per period; a renormalised variation keeps its pre-renormalisation values)
    for (int dmp = 1; dmp < ndt; dmp++) {
        if (!zero_span[dmp]) continue;
        const size_t a = (size_t)(dmp - 1) * n, b = (size_t)dmp * n;
        for (auto *v : {&norm_, &mean_, &disp_, &m2_, &energy_}) std::copy(v->begin() + a, v->begin() + a + n, v->begin() + b);
        if (mbl) std::copy(imb_std.begin() + a, imb_std.begin() + a + n, imb_std.begin() + b);
        std::copy(robs_.begin() + a * nr, robs_.begin() + (a + n) * nr, robs_.begin() + b * nr);
    }
    // MBL spec = <H> / W per trajectory (get_spec_mbl, experiment.cpp:1705-1751): std [dump][tr], lpn
    auto spec_of = [&](const std::vector<std::complex<double>> &src) {
        std::vector<std::complex<double>> out(src.size() / (nr ? nr : 1));
        for (size_t i = 0; i < out.size() && spec; i++)
            out[i] = std::complex<double>(src[i * nr].real() / W, src[i * nr].imag() / W);
        return out;
    };
    const std::vector<std::complex<double>> spec_std = spec_of(robs_), spec_lpn = spec_of(robs_lpn_evo);
    auto write_2d_inv_c = [&](const std::string &fn, const std::vector<std::complex<double>> &v) {
        std::vector<std::complex<double>> inv((size_t)ndt * n);
        for (int dmp = 0; dmp < ndt; dmp++)
            for (int tr = 0; tr < n; tr++) inv[(size_t)tr * ndt + dmp] = v[(size_t)dmp * n + tr];
        save_2d_inv_complex_data(fn, reinterpret_cast<const double *>(inv.data()), ndt, n, 16, false);
    };
    std::vector<double> mean_start(n);
    check(qjx_get_mean_start(h, mean_start.data()), h, "qjx_get_mean_start");
    if (dump_obs == 1 && mbl) {  // MBLCoreBehaviour::dump_std / dump_lpn (core.cpp:4910-4987)
        const size_t o = (size_t)last_dump * n;
        save_double_data(path + "norm" + sfx, norm_.data() + o, n, 16, false);
        save_complex_data(path + "spec" + sfx, reinterpret_cast<const double *>(spec_std.data() + o), n, 16, false);
        save_double_data(path + "imbalance" + sfx, imb_std.data() + o, n, 16, false);
        save_double_data(path + "lambda" + sfx, lam_evo.data() + o, n, 16, false);
        save_int_data(path + "num_renorms" + sfx, renorms.data(), n, false);
        save_complex_data(path + "spec_lpn" + sfx, reinterpret_cast<const double *>(spec_lpn.data() + o), n, 16, false);
        save_double_data(path + "imbalance_lpn" + sfx, mean_lpn_evo.data() + o, n, 16, false);
    }
    if (dump_obs == 1 && integ) {  // IntegrableCoreBehaviour::dump_std / dump_lpn (core.cpp:6685-6753)
        const size_t o = (size_t)last_dump * n;
        save_double_data(path + "norm" + sfx, norm_.data() + o, n, 16, false);
        save_complex_data(path + "spec" + sfx, reinterpret_cast<const double *>(spec_std.data() + o), n, 16, false);
        save_double_data(path + "lambda" + sfx, lam_evo.data() + o, n, 16, false);
        save_int_data(path + "num_renorms" + sfx, renorms.data(), n, false);
        save_complex_data(path + "spec_lpn" + sfx, reinterpret_cast<const double *>(spec_lpn.data() + o), n, 16, false);
    }
    if (dump_obs == 1 && jcs) {  // JCSCoreBehaviour::dump_std / dump_lpn (core.cpp:2976-3033)
        const size_t o = (size_t)last_dump * n;
        save_double_data(path + "norm" + sfx, norm_.data() + o, n, 16, false);
        save_complex_data(path + "spec" + sfx, reinterpret_cast<const double *>(spec_std.data() + o), n, 16, false);
        save_double_data(path + "lambda" + sfx, lam_evo.data() + o, n, 16, false);
        save_int_data(path + "num_renorms" + sfx, renorms.data(), n, false);
        save_complex_data(path + "spec_lpn" + sfx, reinterpret_cast<const double *>(spec_lpn.data() + o), n, 16, false);
        save_double_data(path + "mean" + sfx, mean_lpn_evo.data() + o, n, 16, false);
    }
    if (dump_obs == 1 && !spec) {
        const size_t o = (size_t)last_dump * n;
        save_double_data(path + "norm" + sfx, norm_.data() + o, n, 16, false);  // dump_std
        save_double_data(path + "mean_start" + sfx, mean_start.data(), n, 16, false);
        save_double_data(path + "mean" + sfx, mean_.data() + o, n, 16, false);
        save_double_data(path + "dispersion" + sfx, disp_.data() + o, n, 16, false);
        save_double_data(path + "m2" + sfx, m2_.data() + o, n, 16, false);
        save_double_data(path + "energy" + sfx, energy_.data() + o, n, 16, false);
        const size_t ol = (size_t)last_dump * n;  // dump_lpn
        save_double_data(path + "lambda" + sfx, lam_evo.data() + ol, n, 16, false);
        save_int_data(path + "num_renorms" + sfx, renorms.data(), n, false);
        save_double_data(path + "mean_lpn" + sfx, mean_lpn_evo.data() + ol, n, 16, false);
        save_double_data(path + "energy_lpn" + sfx, energy_lpn_evo.data() + ol, n, 16, false);
    }
    if (dump_obs == 1) {
        if (save_lambdas > 0)
            for (int tr = 0; tr < n; tr++) {
                save_double_vector(path + "delta_f_by_delta_s_" + std::to_string(tr) + sfx, rec_ratio[tr], 16, false);
                save_double_vector(path + "deltas_s_" + std::to_string(tr) + sfx, rec_ds[tr], 16, false);
                save_double_vector(path + "deltas_f_" + std::to_string(tr) + sfx, rec_df[tr], 16, false);
            }
    }
    if (dump_evo_sep == 1 && dump_obs == 1) {
        save_int_data(path + "periods" + sfx, dp.data(), ndt, false);  // dump_std_evo
        write_2d_inv(path + "norm_evo" + sfx, norm_, ndt, ndt, n);
        if (mbl) {  // MBLCoreBehaviour::dump_std_evo (core.cpp:4988-5056)
            write_2d_inv_c(path + "spec_evo" + sfx, spec_std);
            write_2d_inv(path + "imbalance_evo" + sfx, imb_std, ndt, ndt, n);
        } else if (jcs) {  // JCSCoreBehaviour::dump_std_evo (core.cpp:3034-3102): mean = <a^+ a>
            write_2d_inv_c(path + "spec_evo" + sfx, spec_std);
            write_2d_inv(path + "mean_evo" + sfx, energy_, ndt, ndt, n);
        } else if (integ) {  // IntegrableCoreBehaviour::dump_std_evo (core.cpp:6755-6819)
            write_2d_inv_c(path + "spec_evo" + sfx, spec_std);
        } else {
            write_2d_inv(path + "mean_evo" + sfx, mean_, ndt, ndt, n);
            write_2d_inv(path + "dispersion_evo" + sfx, disp_, ndt, ndt, n);
            write_2d_inv(path + "m2_evo" + sfx, m2_, ndt, ndt, n);
            write_2d_inv(path + "energy_evo" + sfx, energy_, ndt, ndt, n);
        }
        auto robs_file = [&](const std::string &name, const std::vector<std::complex<double>> &src) {
            for (int o = 0; o < num_robs; o++) {
                std::vector<std::vector<std::complex<double>>> v(n, std::vector<std::complex<double>>(ndt));
                for (int tr = 0; tr < n; tr++)
                    for (int dmp = 0; dmp < ndt; dmp++) v[tr][dmp] = src[((size_t)dmp * n + tr) * nr + ro + o];
                save_2d_complex_vector(path + name + std::to_string(robs_seed + o) + sfx, v, 16);
            }
        };
        robs_file("random_obs_evo_", robs_);
        if (jump > 0) {
            for (int tr = 0; tr < n; tr++) {
                int64_t k = 0;
                check(qjx_jump_count(h, tr, &k), h, "qjx_jump_count");
                std::vector<double> t(k), nr(k), et(k);
                std::vector<int> ty(k);
                check(qjx_get_jumps(h, tr, t.data(), ty.data(), nr.data(), et.data()), h, "qjx_get_jumps");
                save_double_vector(path + "jump_times_" + std::to_string(tr) + sfx, t, 16, false);
                save_int_vector(path + "diss_types_" + std::to_string(tr) + sfx, ty, false);
                if (jump > 1) {
                    save_double_vector(path + "jump_norms_" + std::to_string(tr) + sfx, nr, 16, false);
                    save_double_vector(path + "jump_etas_" + std::to_string(tr) + sfx, et, 16, false);
                }
            }
        }
        write_2d_inv(path + "lambda_evo" + sfx, lam_evo, ndt, ndt, n);  // dump_lpn_evo
        if (mbl) {  // MBLCoreBehaviour::dump_lpn_evo (core.cpp:5058-5096)
            write_2d_inv_c(path + "spec_lpn_evo" + sfx, spec_lpn);
            write_2d_inv(path + "imbalance_lpn_evo" + sfx, mean_lpn_evo, ndt, ndt, n);
        } else if (jcs) {  // JCSCoreBehaviour::dump_lpn_evo (core.cpp:3104-3150)
            write_2d_inv_c(path + "spec_lpn_evo" + sfx, spec_lpn);
            write_2d_inv(path + "mean_lpn_evo" + sfx, mean_lpn_evo, ndt, ndt, n);
        } else if (integ) {  // IntegrableCoreBehaviour::dump_lpn_evo (core.cpp:6821-6858)
            write_2d_inv_c(path + "spec_lpn_evo" + sfx, spec_lpn);
        } else {
            write_2d_inv(path + "mean_lpn_evo" + sfx, mean_lpn_evo, ndt, ndt, n);
            write_2d_inv(path + "energy_lpn_evo" + sfx, energy_lpn_evo, ndt, ndt, n);
        }
        robs_file("random_obs_lpn_evo_", robs_lpn_evo);
    }
    if (dump_evo_avg == 0) write_adr_avg(last_dump, half, true);

    qjx_stats st{};
    qjx_get_stats(h, &st);
    std::cout << "micro-steps: " << st.micro_steps << ", matvecs: " << st.matvecs
              << ", device time (ms): " << st.kernel_ms << std::endl;
}

}  // namespace

int main(int argc, char **argv)
{
    std::string fn_config = "config.txt", fn_params = "params.txt";
    int device = 0;
    bool check_only = false;
    if (const char *e = std::getenv("QJX_DEVICE")) device = std::atoi(e);
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        if (a == "--config" && i + 1 < argc) fn_config = argv[++i];
        else if (a == "--params" && i + 1 < argc) fn_params = argv[++i];
        else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
        else if (a == "--check") check_only = true;
        else die("unknown argument " + a);
    }

    RunParam rp;
    ConfigParam cp;
    if (!read_config(rp, cp, fn_config)) std::cout << "Unable to open file" << std::endl << "Init with default params" << std::endl;
    if (!read_params(cp, fn_params)) std::cout << "Unable to open file" << std::endl << "Init with default params" << std::endl;
    std::cout << params_echo(rp, cp);

    if (rp.sys_id < 0 || rp.sys_id > 9 || rp.sys_id == 4)
        die("Wrong sys_id: " + std::to_string(rp.sys_id) +
            " (this engine runs the dimer (0), JCS (1), PS (2), MBL (3), Integrable (5), DimerSync (6), Floq2Spins "
            "(7), FloqManySpins (8) and FloqSpinPh (9) systems)");
    const bool jcs = rp.sys_id == 1;  // JCS, MBL, Integrable: Std and LpnMult with the QJ propagator
    const bool mbl = rp.sys_id == 3;
    // Floq2Spins, FloqManySpins: their QJ branch and observables follow the Integrable pattern
    // (spec = <special>)
    const bool floq2 = rp.sys_id == 7, floqn = rp.sys_id == 8, floqp = rp.sys_id == 9;
    const bool integ = rp.sys_id == 5 || floq2 || floqn || floqp;
    const bool ps = rp.sys_id == 2;  // PS: the Std task with the QJ propagator
    const bool dsync = rp.sys_id == 6;
    if (dsync && ((rp.task_id != 1 && rp.task_id != 7) || rp.prop_id != 0))
        die("Wrong task_id / prop_id for sys_id 6 (this engine runs DimerSync with the Std and LpnMult tasks and the "
            "QJ propagator)");
    if (ps && (rp.task_id != 1 || rp.prop_id != 0))
        die("Wrong task_id / prop_id for sys_id 2 (this engine runs PS with the Std task and the QJ propagator)");
    if ((jcs || mbl || integ) && ((rp.task_id != 1 && rp.task_id != 7) || rp.prop_id != 0))
        die("Wrong task_id / prop_id for sys_id " + std::to_string(rp.sys_id) +
            " (this engine runs JCS, MBL and Integrable with the Std and LpnMult tasks and the QJ propagator)");
    if (rp.task_id != 1 && rp.task_id != 4 && rp.task_id != 7 && rp.task_id != 8)
        die("Wrong task_id: " + std::to_string(rp.task_id) +
            " (this engine runs the Std (1), StdDeep (4) and LpnMult (7) tasks)");
    if ((rp.task_id == 4 || rp.task_id == 8) && rp.prop_id != 0)
        die("Wrong prop_id: " + std::to_string(rp.prop_id) + " (StdDeep and LpnMultDeep run the QJ propagator)");
    if (rp.prop_id != 0 && rp.prop_id != 1)
        die("Wrong prop_id: " + std::to_string(rp.prop_id) + " (this engine runs the QJ (0) and RK (1) propagators)");

    try {
        cp.fn_suffix = jcs ? jcs_suffix(rp, cp, 4)
                       : mbl ? mbl_suffix(rp, cp, 4)
                       : floq2 ? floq2spins_suffix(rp, cp, 4)
                       : floqn ? floqnspins_suffix(rp, cp, 4)
                       : floqp ? floqspph_suffix(rp, cp, 4)
                       : integ ? integrable_suffix(rp, cp, 4)
                       : ps    ? ps_suffix(rp, cp, 4)
                       : dsync ? dimersync_suffix(rp, cp, 4)
                               : dimer_suffix(rp, cp, 4);
    } catch (const std::exception &e) {
        die(e.what());
    }
    if (check_only) {
        std::cout << "fn_suffix = " << cp.fn_suffix << std::endl;
        return 0;
    }

    try {
        const bool dimer = !jcs && !mbl && !integ && !ps;
        const int N = (mbl || integ || ps) ? 0 : int(param(cp, dsync ? "dimersync_N" : "N"));
        // PS: 2^ps_num_spins spin states times ps_num_photons_states photon states
        const int ps_ns = ps ? int(param(cp, "ps_num_spins")) : 0, ps_np = ps ? int(param(cp, "ps_num_photons_states")) : 0;
        const int ps_dt = ps ? int(param(cp, "diss_type")) : 0;
        if (ps && (ps_ns < 1 || ps_ns > 8 || ps_np < 2 || (ps_dt != 0 && ps_dt != 1)))
            die("ps_num_spins must be in [1, 8], ps_num_photons_states >= 2, diss_type 0 or 1");
        // Integrable: 2^integrable_N basis states, integrable_N jump channels
        const int Ni = rp.sys_id == 5 ? int(param(cp, "integrable_N")) : 0;
        if (rp.sys_id == 5 && (Ni < 3 || Ni > 10)) die("integrable_N must be in [3, 10]");
        const int nfl = floqn ? int(param(cp, "flqnsp_n")) : 0;
        if (floqn && (nfl < 1 || nfl > 10)) die("flqnsp_n must be in [1, 10]");
        const int nph = floqp ? int(param(cp, "flq_sp_ph_n_ph")) : 0;
        if (floqp && (nph < 1 || nph > 511)) die("flq_sp_ph_n_ph must be in [1, 511]");
        // MBL: C(Nc, Nc/2) basis words and Nc (diss_type 0) or Nc - 1 (diss_type 1) jump channels
        const int Nc = mbl ? int(param(cp, "mbl_Nc")) : 0, mbl_dt = mbl ? int(param(cp, "diss_type")) : 0;
        int d_mbl = 0, nd_mbl = 0;
        if (mbl && qjx_mbl_size(Nc, mbl_dt, &d_mbl, &nd_mbl) != QJX_OK)
            die("mbl_Nc must be even and in [2, 24], diss_type 0 or 1");
        // the dimer has N + 1 Fock states; the JCS oscillator is truncated at N states (newdel.cpp:110)
        const int d = mbl ? d_mbl : floq2 ? 4 : floqn ? (1 << nfl) : floqp ? 2 * (nph + 1) : integ ? (1 << Ni)
                    : ps ? (1 << ps_ns) * ps_np
                    : jcs ? N : N + 1;
        const int n = cp.num_trajectories, deep = cp.ex_deep;
        const int num_diss = mbl ? nd_mbl : floq2 ? 2 : floqn ? nfl : floqp ? 1 : integ ? Ni
                             : ps ? (ps_dt == 0 ? 1 : 1 + ps_ns) : 1;
        // JCS and PS run each drive part as two halves of its tree (init_split_structure_jcs / _ps,
        // core.cpp:10086-10157, 10234-10305: counter 2): four engine branches [K_0, K_0, K_1, K_1]
        // Floq2Spins: one branch of T / 2 per period (init_split_structure_floq2spins)
        const int nbr = (ps || jcs) ? 4 : (floq2 || floqn || floqp) ? 1 : 2;
        const double floq2_T = floq2   ? 2.0 * 3.1415926535897932384626433832795 / param(cp, "flq2sp_freq")
                               : floqn ? 2.0 * 3.1415926535897932384626433832795 / param(cp, "flqnsp_freq")
                               : floqp ? 2.0 * 3.1415926535897932384626433832795 / param(cp, "flq_sp_ph_freq")
                                       : 0.0;
        // DimerSync (newdel.cpp:39-95, 500-563, 2390-2498): the dimer's operators under its own keys,
        // drive 1 in the QJ branches, the period of drive dimersync_main_period
        const int dsync_main = dsync ? int(param(cp, "dimersync_main_period")) : 0;
        if (dsync && dsync_main != 1 && dsync_main != 2) die("Error: wrong dimersync_main_period");
        const double J = dimer ? param(cp, dsync ? "dimersync_prm_J" : "dimer_prm_J") : 0.0;
        const double U = dimer ? param(cp, dsync ? "dimersync_prm_U" : "dimer_prm_U") : 0.0;
        const double E = dimer ? param(cp, dsync ? "dimersync_prm_E" : "dimer_prm_E") : 0.0;
        const double A = dimer ? param(cp, dsync ? "dimersync_drv_ampl_1" : "dimer_drv_ampl") : 0.0;
        const double omega = !dimer ? 1.0
                             : dsync ? param(cp, dsync_main == 1 ? "dimersync_drv_freq_1" : "dimersync_drv_freq_2")
                                     : param(cp, "dimer_drv_freq");
        const double mbl_W = mbl ? param(cp, "mbl_prm_W") : 1.0;
        const double g = param(cp, "diss_gamma");
        const double jcs_alpha = jcs ? param(cp, "jcs_prm_alpha") : 0.0;
        const double jcs_ampl = jcs ? param(cp, "jcs_drv_ampl") : 0.0;
        const double jcs_p1 = jcs ? param(cp, "jcs_drv_part_1") : 0.0, jcs_p2 = jcs ? param(cp, "jcs_drv_part_2") : 0.0;
        const int start_type = int(param(cp, "start_type")), start_state = int(param(cp, "start_state"));
        const int jump = int(param(cp, "jump"));
        const int dump_obs = int(param(cp, "dump_obs")), dump_evo_sep = int(param(cp, "dump_evo_sep"));
        const int dump_evo_avg = int(param(cp, "dump_evo_avg")), dump_adr_sep = int(param(cp, "dump_adr_sep"));
        const int dump_adr_avg_on = int(param(cp, "dump_adr_avg"));
        const int dump_phi_on = int(param(cp, "dump_phi")), dump_phi_evo_on = int(param(cp, "dump_phi_evo"));
        const int jumps_counts_lim = int(param(cp, "jumps_counts"));
        // optional key (no counterpart in QJX): ensemble purity per dump into purity_evo
        const int dump_purity = int(param_or(cp, "dump_purity", 0));
        const int num_robs = int(param(cp, "num_random_obs"));
        const int robs_seed = int(param_or(cp, "random_obs_seed", 0));
        if (n < 1 || (dimer && N < 1) || (jcs && N < 2)) die("num_trajectories and N must be positive (N >= 2 for JCS)");
        if (start_type == 0 && (start_state < 0 || start_state >= d)) die("start_state out of range");
        const std::string &sfx = cp.fn_suffix;
        const std::string path = rp.path;
        const size_t dd = (size_t)d * d;

        // model (newdel.cpp init_*), debug dumps (debugger.cpp:142-168, qj_proc.cpp:115-119)
        std::vector<double> H(2 * dd), Hd(2 * dd), L(2 * dd * num_diss), K(4 * dd), Ut(2 * dd * deep * nbr);
        std::vector<double> Sps(ps ? 8 * dd : 0);  // PS: special, special_2, special_3, special_4
        const double ps_alpha = ps ? param(cp, "ps_prm_alpha") : 0.0;
        const double ps_p1 = ps ? param(cp, "ps_drv_part_1") : 0.0, ps_p2 = ps ? param(cp, "ps_drv_part_2") : 0.0;
        // StdDeep (task_id 4): the split tree of the sub-period T / (2 deep_num_steps)
        const bool deep_task = rp.task_id == 4 || rp.task_id == 8;  // StdDeep, LpnMultDeep
        const int nsub = deep_task ? int(param(cp, "deep_num_steps")) : 0;
        if (deep_task && nsub < 1) die("deep_num_steps must be positive");
        // JCS: the number operator (energy slot) and a = special (first random-observable slot)
        std::vector<double> Nop(jcs ? 2 * dd : 0), Aop(jcs ? 2 * dd : 0);
        if (jcs)
            check(qjx_build_jcs(N, jcs_alpha, jcs_ampl, jcs_p1, jcs_p2, deep, H.data(), Hd.data(), L.data(), Nop.data(),
                                Aop.data(), K.data(), Ut.data()),
                  nullptr, "qjx_build_jcs");
        if (jcs) {  // engine branches [U_0, U_0, U_1, U_1]
            const size_t tree = 2 * dd * deep;
            std::copy(Ut.begin() + tree, Ut.begin() + 2 * tree, Ut.begin() + 2 * tree);
            std::copy(Ut.begin() + 2 * tree, Ut.begin() + 3 * tree, Ut.begin() + 3 * tree);
            std::copy(Ut.begin(), Ut.begin() + tree, Ut.begin() + tree);
        } else if (mbl) {
            // one branch head of duration mbl_T with two children of the same split tree
            // (init_split_structure_mbl, core.cpp:10382-10432): the engine's two branches
            std::vector<double> en(Nc);
            check(qjx_build_mbl(Nc, mbl_W, param(cp, "mbl_prm_U"), param(cp, "mbl_prm_J"), int(param(cp, "mbl_seed")),
                                int(param(cp, "mbl_mns")), mbl_dt, param(cp, "diss_phase"), g, param(cp, "mbl_T"),
                                deep, en.data(), nullptr, H.data(), L.data(), K.data(), Ut.data()),
                  nullptr, "qjx_build_mbl");
            std::copy(Ut.begin(), Ut.begin() + 2 * dd * deep, Ut.begin() + 2 * dd * deep);
            std::copy(K.begin(), K.begin() + 2 * dd, K.begin() + 2 * dd);
            // written to the working directory, without `path` (newdel.cpp:903-905)
            save_double_data("energies" + cp.fn_suffix, en.data(), Nc, 16, false);
        } else if (ps) {
            check(qjx_build_ps(ps_ns, ps_np, ps_alpha, param(cp, "ps_prm_d"), param(cp, "ps_prm_g"),
                               param(cp, "ps_drv_ampl"), ps_dt, param(cp, "ps_diss_w"), ps_p1, ps_p2, deep, H.data(),
                               Hd.data(), L.data(), Sps.data(), K.data(), Ut.data()),
                  nullptr, "qjx_build_ps");
            // engine branches [U_0, U_0, U_1, U_1]
            const size_t tree = 2 * dd * deep;
            std::copy(Ut.begin() + tree, Ut.begin() + 2 * tree, Ut.begin() + 2 * tree);
            std::copy(Ut.begin() + 2 * tree, Ut.begin() + 3 * tree, Ut.begin() + 3 * tree);
            std::copy(Ut.begin(), Ut.begin() + tree, Ut.begin() + tree);
        } else if (floq2) {  // H is also the special (spec) matrix: a copy into Hd's storage
            check(qjx_build_floq2spins(param(cp, "flq2sp_Delta_1"), param(cp, "flq2sp_Delta_2"), param(cp, "flq2sp_J"),
                                       param(cp, "flq2sp_gamma"), floq2_T, deep, H.data(), L.data(), K.data(),
                                       Ut.data()),
                  nullptr, "qjx_build_floq2spins");
            Hd = H;
        } else if (floqp) {  // as Floq2Spins, for a spin and a photon mode
            check(qjx_build_floqspph(nph, param(cp, "flq_sp_ph_Delta"), param(cp, "flq_sp_ph_Omega"),
                                     param(cp, "flq_sp_ph_gamma"), floq2_T, deep, H.data(), L.data(), K.data(), Ut.data()),
                  nullptr, "qjx_build_floqspph");
            Hd = H;
        } else if (floqn) {  // as Floq2Spins, for n spins
            check(qjx_build_floqnspins(nfl, param(cp, "flqnsp_Delta"), param(cp, "flqnsp_J"), param(cp, "flqnsp_gamma"),
                                       floq2_T, deep, H.data(), L.data(), K.data(), Ut.data()),
                  nullptr, "qjx_build_floqnspins");
            Hd = H;
        } else if (integ) {
            // H = 0; `special` (the spec observable) into Hd's storage; one head of duration
            // integrable_T with two children of the same split tree (init_split_structure_integrable)
            check(qjx_build_integrable(Ni, int(param(cp, "integrable_seed")), int(param(cp, "integrable_num_seeds")),
                                       param(cp, "integrable_tau"), param(cp, "integrable_k"), param(cp, "integrable_T"),
                                       deep, L.data(), Hd.data(), K.data(), Ut.data()),
                  nullptr, "qjx_build_integrable");
            std::copy(Ut.begin(), Ut.begin() + 2 * dd * deep, Ut.begin() + 2 * dd * deep);
            std::copy(K.begin(), K.begin() + 2 * dd, K.begin() + 2 * dd);
        }
        else if (deep_task)
            check(qjx_build_dimer_deep(N, J, U, E, A, g, omega, deep, nsub, H.data(), Hd.data(), L.data(), K.data(),
                                       Ut.data()),
                  nullptr, "qjx_build_dimer_deep");
        else
            check(qjx_build_dimer(N, J, U, E, A, g, omega, deep, H.data(), Hd.data(), L.data(), K.data(), Ut.data()),
                  nullptr, "qjx_build_dimer");
        std::cout << "init_sizes" << std::endl << "init_hamiltonians" << std::endl << "init_dissipators" << std::endl
                  << "init_hamiltonians_qj" << std::endl;
        if (rp.is_debug && (mbl || integ)) {  // MBL / IntegrableDebugBehaviour::save (debugger.cpp:55-95)
            save_complex_data(path + "hamiltonian" + sfx, H.data(), dd, 16, false);
            for (int c = 0; c < num_diss; c++)
                save_complex_data(path + "dissipator_" + std::to_string(c) + sfx, L.data() + 2 * dd * c, dd, 16, false);
            save_complex_data(path + "hamiltonians_qj_0" + sfx, K.data(), dd, 16, false);
            save_complex_data(path + "spec_mtx" + sfx, integ ? Hd.data() : H.data(), dd, 16, false);
            save_complex_data(path + "exp_mtx_0" + sfx, Ut.data() + 2 * dd * (deep - 1), dd, 16, false);
        } else if (rp.is_debug) {  // Dimer / JCS / PSDebugBehaviour::save (debugger.cpp:3-53)
            save_complex_data(path + "hamiltonian" + sfx, H.data(), dd, 16, false);
            for (int c = 0; c < num_diss; c++)
                save_complex_data(path + "dissipator_" + std::to_string(c) + sfx, L.data() + 2 * dd * c, dd, 16, false);
            for (int b = 0; b < 2; b++) {
                save_complex_data(path + "hamiltonians_qj_" + std::to_string(b) + sfx, K.data() + 2 * dd * b, dd, 16, false);
                if (rp.prop_id == 0)  // the split tree exists for the QJ propagator only (qj_proc.cpp:115-119)
                    save_complex_data(path + "exp_mtx_" + std::to_string(b) + sfx,
                                      Ut.data() + 2 * dd * ((size_t)((ps || jcs) ? 2 * b : b) * deep + deep - 1), dd, 16,
                                      false);
            }
            if (jcs) save_complex_data(path + "spec_mtx" + sfx, Aop.data(), dd, 16, false);
            if (ps) {
                const char *names[4] = {"spec_mtx", "spec_2_mtx", "spec_3_mtx", "spec_4_mtx"};
                for (int o = 0; o < 4; o++) save_complex_data(path + names[o] + sfx, Sps.data() + 2 * dd * o, dd, 16, false);
            }
        }
        std::vector<double> HE(2 * dd);
        for (size_t e = 0; e < 2 * dd; e++) HE[e] = jcs ? Nop[e] : (mbl || integ || ps) ? H[e] : H[e] + E * Hd[e];
        std::vector<double> R =
            random_observables(d, num_robs, robs_seed, int(param_or(cp, "random_obs_mns", 1000000)),
                               int(param_or(cp, "random_obs_type", 0)));
        // JCS: spec = <a> / alpha, MBL: spec = <H> / W ride in observable slot 0
        // Integrable: spec = <special> rides in observable slot 0 as well
        // PS: spec, spec_2, spec_3 and the photon number ride in slots 0..3
        const int robs_off = (jcs || mbl || integ) ? 1 : ps ? 4 : 0;
        if (jcs) R.insert(R.begin(), Aop.begin(), Aop.end());
        if (mbl) R.insert(R.begin(), H.begin(), H.end());
        if (integ) R.insert(R.begin(), Hd.begin(), Hd.end());
        if (ps) R.insert(R.begin(), Sps.begin(), Sps.end());
        const int nr_eng = num_robs + robs_off;

        // dump schedule (init_dump_periods)
        // StdDeep: a dump after every sub-period, labelled with its period (init_dump_periods_deep,
        // newdel_exp.cpp:377-406)
        std::vector<int> dp;
        if (deep_task) {
            dp.push_back(0);
            for (int p = 0; p < cp.num_obs_periods; p++)
                for (int k = 0; k < 2 * nsub; k++) dp.push_back(p);
        } else {
            dp = dump_periods(int(param(cp, "dump_type")), int(param(cp, "dump_num")), cp.num_obs_periods);
        }
        if (dp.empty()) die("Wrong dump_type");
        const int ndt = (int)dp.size();
        bool increasing = true;
        for (int i = 1; i < ndt; i++) increasing = increasing && dp[i] > dp[i - 1];

        qjx_config cfg{};
        cfg.d = d;
        cfg.n_traj = n;
        cfg.deep = deep;
        cfg.num_branches = nbr;
        cfg.num_diss = num_diss;
        cfg.num_robs = nr_eng;
        cfg.T = jcs     ? jcs_alpha
                : ps    ? ps_alpha
                : mbl   ? param(cp, "mbl_T")
                : (floq2 || floqn || floqp) ? floq2_T
                : integ ? param(cp, "integrable_T")
                        : 2.0 * 3.1415926535897932384626433832795 / omega;
        // JCS: part b's head is jcs_drv_part_b * alpha, run as two halves (init_split_structure_jcs,
        // core.cpp:10086-10157)
        const double jcs_len[4] = {0.5 * (jcs_p1 * jcs_alpha), 0.5 * (jcs_p1 * jcs_alpha), 0.5 * (jcs_p2 * jcs_alpha),
                                   0.5 * (jcs_p2 * jcs_alpha)};
        // PS: part b (head part_b alpha) as two halves (init_split_structure_ps, core.cpp:10234-10305)
        const double ps_len[4] = {0.5 * (ps_p1 * ps_alpha), 0.5 * (ps_p1 * ps_alpha), 0.5 * (ps_p2 * ps_alpha),
                                  0.5 * (ps_p2 * ps_alpha)};
        cfg.branch_len = jcs ? jcs_len : ps ? ps_len : nullptr;
        cfg.record = jump;
        cfg.rng_kind = int(param_or(cp, "rng_kind", 0));
        cfg.seed = (uint64_t)(uint32_t)cp.seed;
        cfg.rec_cap = 1024;
        // MBL: the imbalance of every recorded dump comes from its adr rows
        cfg.keep_adr = ((dump_evo_sep == 1 && dump_adr_sep == 1) || dump_evo_avg == 1 || mbl) ? 1 : 0;
        cfg.max_dumps = ndt;
        cfg.deep_num_steps = nsub;
        cfg.device = device;
        const std::vector<double> gr(num_diss, 1.0);  // head->g (core.cpp:9905, 10418)
        qjx_engine *h = nullptr;
        if (rp.prop_id == 0) {
            check(qjx_create(&cfg, Ut.data(), L.data(), gr.data(), HE.data(), nr_eng ? R.data() : nullptr, &h), nullptr,
                  "qjx_create");
        } else {  // RK propagator: rk_right_part_dimer's drive keys (core.cpp:11048-11051)
            std::vector<double> He(2 * dd), Hdr(2 * dd);
            check(qjx_build_dimer_rk(N, J, U, E, g, He.data(), Hdr.data()), nullptr, "qjx_build_dimer_rk");
            check(qjx_create_rk(&cfg, He.data(), Hdr.data(), E, A, int(param_or(cp, "dimer_drv_type", 0)), omega,
                                param_or(cp, "dimer_drv_phase", 0.0), cp.rk_ns, L.data(), gr.data(), HE.data(),
                                num_robs ? R.data() : nullptr, &h),
                  nullptr, "qjx_create_rk");
        }

        // init_data: start states (newdel_exp.cpp:656-679)
        std::vector<double> psi(2 * (size_t)n * d, 0.0);
        for (int tr = 0; tr < n; tr++)
            for (int i = 0; i < d; i++)
                if (start_type == 0) psi[2 * ((size_t)tr * d + i)] = (i == start_state) ? 1.0 : 0.0;
                else psi[2 * ((size_t)tr * d + i)] = std::sqrt(1.0 / double(d));
        check(qjx_set_states(h, psi.data()), h, "qjx_set_states");
        std::cout << "init_data" << std::endl;

        if (rp.task_id == 7 || rp.task_id == 8) {
            // DimerSync's Lyapunov characteristics are the dimer's (DimerSyncCoreBehaviour, core.cpp:1812-1997)
            // Floq2Spins's are the Integrable ones (spec only; core.cpp:7546-7690)
            run_lpn_mult(h, rp, cp, cfg, H, d, num_robs, robs_seed, dsync ? 0 : (floq2 || floqn || floqp) ? 5 : rp.sys_id, Nc, jcs ? jcs_alpha : mbl ? mbl_W : 1.0,
                         jcs ? jcs_p1 * jcs_alpha + jcs_p2 * jcs_alpha : cfg.T, nsub);
            qjx_destroy(h);
            return 0;
        }

        // trans_process (experiment.cpp:411-446)
        check(qjx_init_thresholds(h), h, "qjx_init_thresholds");
        check(qjx_run_periods(h, cp.num_tp_periods, 0, nullptr, 0, 0), h, "qjx_run_periods");
        check(qjx_reset_times(h), h, "qjx_reset_times");
        check(qjx_observe(h, 0, 1), h, "qjx_observe");

        auto get_adr = [&](int dump) {
            std::vector<double> adr((size_t)n * d);
            if (cfg.keep_adr) check(qjx_get_observables(h, dump, 1, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                                        adr.data()), h, "qjx_get_observables");
            else check(qjx_get_observables(h, 0, 1, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, adr.data()),
                       h, "qjx_get_observables");
            return adr;
        };
        auto write_adr_single = [&](int dump, bool append) {  // dump_adr_single (dump.cpp:3-24)
            if (!(dump_evo_sep == 1 && dump_adr_sep == 1)) return;
            const std::vector<double> adr = get_adr(dump);
            for (int tr = 0; tr < n; tr++)
                save_double_data(path + "adr_" + std::to_string(tr) + sfx, adr.data() + (size_t)tr * d, d, 16, append);
        };
        auto write_adr_avg = [&](int dump, bool append) {  // dump_adr_avg (dump.cpp:26-61)
            if (dump_adr_avg_on != 1) return;
            const std::vector<double> adr = get_adr(dump);
            std::vector<double> avg(d, 0.0);
            for (int tr = 0; tr < n; tr++)
                for (int st = 0; st < d; st++) avg[st] += adr[(size_t)tr * d + st] / double(n);
            save_double_data(path + "adr_avg" + sfx, avg.data(), d, 16, append);
        };
        auto write_phi = [&](const std::string &prefix, bool append) {  // dump_phi / dump_phi_evo
            check(qjx_get_states(h, psi.data(), nullptr, nullptr, nullptr), h, "qjx_get_states");
            for (int tr = 0; tr < n; tr++)
                save_complex_data(path + prefix + std::to_string(tr) + sfx, psi.data() + 2 * (size_t)tr * d, d, 16, append);
        };
        std::vector<double> purity_evo;
        auto take_purity = [&]() {
            if (dump_purity != 1) return;
            double p = 0.0;
            check(qjx_purity(h, &p, nullptr), h, "qjx_purity");
            purity_evo.push_back(p);
        };
        take_purity();
        write_adr_single(0, false);
        if (dump_evo_avg == 1) write_adr_avg(0, false);

        // obser_process (experiment.cpp:448-542)
        if (dump_phi_evo_on == 1 && !deep_task) write_phi("phi_evo_", false);
        int last_dump = 0;
        const bool per_interval = jumps_counts_lim > 0 || !increasing || dump_phi_evo_on == 1 ||
                                  (dump_evo_sep == 1 && dump_adr_sep == 1) || dump_evo_avg == 1 || rp.is_pp == 1 ||
                                  dump_purity == 1;
        if (deep_task) {
            // StdDeep obser_process (experiment.cpp:806-845): a period per step, observables after
            // every sub-period inside it, adr files per sub-period, adr_avg per period
            const int per_period = 2 * nsub;
            for (int p = 0; p < cp.num_obs_periods; p++) {
                if (rp.is_pp == 1) std::cout << "dump_id: " << p + 1 << std::endl;
                check(qjx_run_periods(h, 1, 1, nullptr, 0, 1 + p * per_period), h, "qjx_run_periods");
                for (int k = 0; k < per_period; k++) write_adr_single(1 + p * per_period + k, true);
                if (dump_evo_avg == 1) write_adr_avg(per_period * (p + 1), true);
            }
            last_dump = ndt - 1;
        } else if (!per_interval) {
            // one call: every trajectory runs all observation periods, observables at each dump
            std::vector<int> at(dp.begin() + 1, dp.end());
            if (ndt > 1) check(qjx_run_periods(h, dp[ndt - 1], 1, at.data(), ndt - 1, 1), h, "qjx_run_periods");
            last_dump = ndt - 1;
        } else {
            std::vector<int> jc(n);
            bool finished = false;
            for (int dump_id = 1; dump_id < ndt && !finished; dump_id++) {
                if (rp.is_pp == 1) std::cout << "dump_id: " << dump_id << std::endl;
                const int span = dp[dump_id] - dp[dump_id - 1];
                if (jumps_counts_lim > 0) {
                    for (int p = 0; p < span; p++) {
                        check(qjx_run_periods(h, 1, 1, nullptr, 0, 0), h, "qjx_run_periods");
                        check(qjx_get_states(h, nullptr, nullptr, nullptr, jc.data()), h, "qjx_get_states");
                        bool all = true;
                        for (int tr = 0; tr < n; tr++) all = all && jc[tr] >= jumps_counts_lim;
                        if (all) {
                            finished = true;
                            break;
                        }
                    }
                    check(qjx_observe(h, dump_id, 0), h, "qjx_observe");
                } else if (span > 0) {
                    const int at = span;
                    check(qjx_run_periods(h, span, 1, &at, 1, dump_id), h, "qjx_run_periods");
                } else {
                    check(qjx_observe(h, dump_id, 0), h, "qjx_observe");
                }
                last_dump = dump_id;
                take_purity();
                write_adr_single(dump_id, true);
                if (dump_phi_evo_on == 1) write_phi("phi_evo_", true);
                if (dump_evo_avg == 1) write_adr_avg(dump_id, true);
            }
        }
        const int nrec = last_dump + 1;
        if (dump_purity == 1) save_double_data(path + "purity_evo" + sfx, purity_evo.data(), purity_evo.size(), 16, false);

        // collect observables of the recorded dumps
        Dumps D;
        const size_t nd_ = (size_t)nrec * n;
        D.norm.assign(nd_, 0.0);
        D.mean.assign(nd_, 0.0);
        D.disp.assign(nd_, 0.0);
        D.m2.assign(nd_, 0.0);
        D.energy.assign(nd_, 0.0);
        D.robs.assign(nd_ * (nr_eng ? nr_eng : 1), 0.0);
        check(qjx_get_observables(h, 0, nrec, D.norm.data(), D.mean.data(), D.disp.data(), D.m2.data(), D.energy.data(),
                                  nr_eng ? reinterpret_cast<double *>(D.robs.data()) : nullptr, nullptr),
              h, "qjx_get_observables");
        // JCS: spec = <a> / alpha (get_spec_jcs, experiment.cpp:1520-1562), mean = <a^+ a>
        // (get_num_photons_jcs, experiment.cpp:2080-2160) from the energy slot
        // MBL: spec = <H> / W (get_spec_mbl, experiment.cpp:1705-1751), imbalance from the adr rows
        // (get_imbalance_mbl, experiment.cpp:1753-1800)
        std::vector<std::complex<double>> spec((jcs || mbl || integ || ps) ? nd_ : 0);
        // get_spec_integrable: no division; get_spec_ps (experiment.cpp:1568-1614): / alpha
        const double spec_div = jcs ? jcs_alpha : mbl ? mbl_W : ps ? ps_alpha : 1.0;
        for (size_t i = 0; i < spec.size(); i++) {
            const std::complex<double> a = D.robs[i * nr_eng];
            spec[i] = std::complex<double>(a.real() / spec_div, a.imag() / spec_div);
        }
        // PS: spec_2 = <J_z>, spec_3 = <J_+>, mean = Re <a^+ a> (get_spec_2_ps, get_spec_3_ps,
        // get_num_photons_ps, experiment.cpp:1616-1708, 2170-2216) from slots 1, 2, 3
        std::vector<std::complex<double>> spec2(ps ? nd_ : 0), spec3(ps ? nd_ : 0);
        std::vector<double> ps_mean(ps ? nd_ : 0);
        for (size_t i = 0; i < spec2.size(); i++) {
            spec2[i] = D.robs[i * nr_eng + 1];
            spec3[i] = D.robs[i * nr_eng + 2];
            ps_mean[i] = D.robs[i * nr_eng + 3].real();
        }
        std::vector<double> imbalance(mbl ? nd_ : 0);
        if (mbl) {
            std::vector<double> adr(nd_ * d);
            check(qjx_get_observables(h, 0, nrec, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, adr.data()), h,
                  "qjx_get_observables");
            check(qjx_mbl_imbalance(Nc, int(nd_), adr.data(), imbalance.data()), h, "qjx_mbl_imbalance");
        }
        std::vector<double> mean_start(n);
        check(qjx_get_mean_start(h, mean_start.data()), h, "qjx_get_mean_start");

        if (ps && dump_obs == 1) {  // PSCoreBehaviour::dump_std (core.cpp:3958-3995)
            const size_t o = (size_t)last_dump * n;
            save_double_data(path + "norm" + sfx, D.norm.data() + o, n, 16, false);
            save_complex_data(path + "spec" + sfx, reinterpret_cast<const double *>(spec.data() + o), n, 16, false);
            save_complex_data(path + "spec_2" + sfx, reinterpret_cast<const double *>(spec2.data() + o), n, 16, false);
            save_complex_data(path + "spec_3" + sfx, reinterpret_cast<const double *>(spec3.data() + o), n, 16, false);
            save_double_data(path + "mean" + sfx, ps_mean.data() + o, n, 16, false);
        }
        if (mbl && dump_obs == 1) {  // MBLCoreBehaviour::dump_std (core.cpp:4910-4937)
            const size_t o = (size_t)last_dump * n;
            save_double_data(path + "norm" + sfx, D.norm.data() + o, n, 16, false);
            save_complex_data(path + "spec" + sfx, reinterpret_cast<const double *>(spec.data() + o), n, 16, false);
            save_double_data(path + "imbalance" + sfx, imbalance.data() + o, n, 16, false);
        }
        if ((jcs || integ) && dump_obs == 1) {  // JCS / Integrable dump_std (core.cpp:2976-2999, 6685-6708)
            const size_t o = (size_t)last_dump * n;
            save_double_data(path + "norm" + sfx, D.norm.data() + o, n, 16, false);
            save_complex_data(path + "spec" + sfx, reinterpret_cast<const double *>(spec.data() + o), n, 16, false);
        }
        // dump_std (core.cpp:918-957): values of the last dump
        if (dimer && dump_obs == 1) {
            const size_t o = (size_t)last_dump * n;
            save_double_data(path + "norm" + sfx, D.norm.data() + o, n, 16, false);
            save_double_data(path + "mean_start" + sfx, mean_start.data(), n, 16, false);
            save_double_data(path + "mean" + sfx, D.mean.data() + o, n, 16, false);
            save_double_data(path + "dispersion" + sfx, D.disp.data() + o, n, 16, false);
            save_double_data(path + "m2" + sfx, D.m2.data() + o, n, 16, false);
            save_double_data(path + "energy" + sfx, D.energy.data() + o, n, 16, false);
        }
        if (dump_phi_on == 1 && !deep_task) write_phi("phi_", false);
        if (dump_phi_evo_on == 1 && !deep_task) write_phi("phi_evo_", true);

        // dump_std_evo (core.cpp:1008-1084): rows = dumps, columns = trajectories
        if (dump_evo_sep == 1 && dump_obs == 1) {
            save_int_data(path + "periods" + sfx, dp.data(), ndt, false);
            std::vector<double> inv((size_t)ndt * n, 0.0);  // [tr][dump] like ed->*_evo
            auto evo = [&](const std::vector<double> &v, const char *name) {
                for (int dmp = 0; dmp < nrec; dmp++)
                    for (int tr = 0; tr < n; tr++) inv[(size_t)tr * ndt + dmp] = v[(size_t)dmp * n + tr];
                save_2d_inv_double_data(path + name + sfx, inv.data(), ndt, n, 16, false);
            };
            evo(D.norm, "norm_evo");
            if (jcs || mbl || integ || ps) {  // dump_std_evo (core.cpp:3034-3102, 4052-4130, 4988-5056, 6755-6819)
                auto cevo = [&](const std::vector<std::complex<double>> &v, const char *name) {
                    std::vector<std::complex<double>> cinv((size_t)ndt * n);
                    for (int dmp = 0; dmp < nrec; dmp++)
                        for (int tr = 0; tr < n; tr++) cinv[(size_t)tr * ndt + dmp] = v[(size_t)dmp * n + tr];
                    save_2d_inv_complex_data(path + name + sfx, reinterpret_cast<const double *>(cinv.data()), ndt, n,
                                             16, false);
                };
                cevo(spec, "spec_evo");
                if (ps) {
                    cevo(spec2, "spec_2_evo");
                    cevo(spec3, "spec_3_evo");
                    evo(ps_mean, "mean_evo");
                }
                if (jcs) evo(D.energy, "mean_evo");
                else if (mbl) evo(imbalance, "imbalance_evo");
            } else {
                evo(D.mean, "mean_evo");
                evo(D.disp, "dispersion_evo");
                evo(D.m2, "m2_evo");
                evo(D.energy, "energy_evo");
            }
            for (int o = 0; o < num_robs; o++) {
                std::vector<std::vector<std::complex<double>>> v(n, std::vector<std::complex<double>>(nrec));
                for (int tr = 0; tr < n; tr++)
                    for (int dmp = 0; dmp < nrec; dmp++)
                        v[tr][dmp] = D.robs[((size_t)dmp * n + tr) * nr_eng + robs_off + o];
                save_2d_complex_vector(path + "random_obs_evo_" + std::to_string(robs_seed + o) + sfx, v, 16);
            }
            if (jump > 0) {
                for (int tr = 0; tr < n; tr++) {
                    int64_t k = 0;
                    check(qjx_jump_count(h, tr, &k), h, "qjx_jump_count");
                    std::vector<double> t(k), nr(k), et(k);
                    std::vector<int> ty(k);
                    check(qjx_get_jumps(h, tr, t.data(), ty.data(), nr.data(), et.data()), h, "qjx_get_jumps");
                    save_double_vector(path + "jump_times_" + std::to_string(tr) + sfx, t, 16, false);
                    save_int_vector(path + "diss_types_" + std::to_string(tr) + sfx, ty, false);
                    if (jump > 1) {
                        save_double_vector(path + "jump_norms_" + std::to_string(tr) + sfx, nr, 16, false);
                        save_double_vector(path + "jump_etas_" + std::to_string(tr) + sfx, et, 16, false);
                    }
                }
            }
        }
        if (dump_evo_avg == 0) write_adr_avg(last_dump, false);

        qjx_stats st{};
        qjx_get_stats(h, &st);
        std::cout << "micro-steps: " << st.micro_steps << ", matvecs: " << st.matvecs
                  << ", device time (ms): " << st.kernel_ms << std::endl;
        qjx_destroy(h);
    } catch (const std::exception &e) {
        die(e.what());
    }
    return 0;
}
