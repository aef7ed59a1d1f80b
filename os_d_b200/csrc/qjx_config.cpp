// qjx_config.cpp -- parameter files, file-name suffix, dump schedule and output writers with
// the formats of the reference (source/cpp/QJX/QJX/config.cpp, outputter.cpp, utils.cpp,
// newdel_exp.cpp:408-455, newdel.cpp:3652-3750).
#include "qjx_config.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <stdexcept>

namespace qjxio {

// Tokens of a config.txt line: the pieces of `str` between occurrences of `delim`, with empty
// pieces dropped.  A run of delimiters, or one at either end, therefore yields no token, while
// any other character (a tab, a trailing carriage return) stays inside its token.  This is the
// tokenisation of the reference's reader (QJX/config.cpp:3-27, used at :109-114).
std::vector<std::string> split(const std::string &str, const std::string &delim)
{
    std::vector<std::string> out;
    if (delim.empty()) {
        if (!str.empty()) out.push_back(str);
        return out;
    }
    std::string::size_type start = 0;
    for (;;) {
        const std::string::size_type hit = str.find(delim, start);
        const std::string::size_type stop = (hit == std::string::npos) ? str.size() : hit;
        if (stop > start) out.emplace_back(str, start, stop - start);
        if (hit == std::string::npos) return out;
        start = hit + delim.size();
    }
}

void set_param(RunParam &rp, ConfigParam &cp, const std::string &k, const std::string &v)
{
    const int iv = std::atoi(v.c_str());
    if (k == "sys_id") rp.sys_id = iv;
    if (k == "task_id") rp.task_id = iv;
    if (k == "prop_id") rp.prop_id = iv;
    if (k == "is_debug") rp.is_debug = iv;
    if (k == "is_pp") rp.is_pp = iv;
    if (k == "init_fn") rp.init_fn = v;
    if (k == "path") rp.path = v;
    if (k == "num_threads") rp.num_threads = iv;
    if (k == "num_trajectories") cp.num_trajectories = iv;
    if (k == "seed") cp.seed = iv;
    if (k == "mns") cp.mns = iv;
    if (k == "num_tp_periods") cp.num_tp_periods = iv;
    if (k == "num_obs_periods") cp.num_obs_periods = iv;
    if (k == "ex_deep") cp.ex_deep = iv;
    if (k == "rk_ns") cp.rk_ns = iv;
}

bool read_config(RunParam &rp, ConfigParam &cp, const std::string &fn)
{
    std::ifstream f(fn);
    if (!f.is_open()) return false;
    std::string line;
    while (std::getline(f, line)) {
        const std::vector<std::string> t = split(line, " ");
        if (t.size() == 2) set_param(rp, cp, t[0], t[1]);
    }
    return true;
}

bool read_params(ConfigParam &cp, const std::string &fn)
{
    std::ifstream f(fn);
    if (!f.is_open()) return false;
    std::string line, key;
    double val = 0.0;
    while (std::getline(f, line)) {
        std::istringstream iss(line);
        iss >> key >> val;
        cp.params[key] = val;
    }
    return true;
}

std::string params_echo(const RunParam &rp, const ConfigParam &cp)
{
    std::ostringstream o;
    o << "############# parameters #############" << std::endl;
    o << "sys_id = " << rp.sys_id << std::endl;
    o << "task_id = " << rp.task_id << std::endl;
    o << "prop_id = " << rp.prop_id << std::endl;
    o << "is_debug = " << rp.is_debug << std::endl;
    o << "is_pp = " << rp.is_pp << std::endl;
    o << "init_fn = " << rp.init_fn << std::endl;
    o << "path = " << rp.path << std::endl;
    o << "num_threads = " << rp.num_threads << std::endl;
    o << "num_trajectories = " << cp.num_trajectories << std::endl;
    o << "seed = " << cp.seed << std::endl;
    o << "mns = " << cp.mns << std::endl;
    o << "num_tp_periods = " << cp.num_tp_periods << std::endl;
    o << "num_obs_periods = " << cp.num_obs_periods << std::endl;
    o << "ex_deep = " << cp.ex_deep << std::endl;
    o << "rk_ns = " << cp.rk_ns << std::endl;
    o << std::endl;
    for (const auto &kv : cp.params) o << kv.first << ": " << kv.second << std::endl;
    o << "######################################" << std::endl;
    return o.str();
}

double param(const ConfigParam &cp, const std::string &key)
{
    auto it = cp.params.find(key);
    if (it == cp.params.end()) throw std::runtime_error("missing key in params file: " + key);
    return it->second;
}

double param_or(const ConfigParam &cp, const std::string &key, double dflt)
{
    auto it = cp.params.find(key);
    return it == cp.params.end() ? dflt : it->second;
}

static std::string lpn_suffix(const RunParam &rp, const ConfigParam &cp)
{
    if (rp.task_id != 7 && rp.task_id != 8) return "";
    std::stringstream p;  // suffix_lpn (outputter.cpp:371-381)
    p << "_lpn(" << std::defaultfloat << std::setprecision(6) << param(cp, "lpn_type") << "_" << std::setprecision(4)
      << std::fixed << std::log10(param(cp, "lpn_delta_s")) << "_" << std::setprecision(4) << std::fixed
      << std::log10(param(cp, "lpn_delta_f_high")) << "_" << std::setprecision(4) << std::fixed
      << std::log10(param(cp, "lpn_delta_f_low")) << ")";
    return p.str();
}

std::string dimer_suffix(const RunParam &rp, const ConfigParam &cp, int precision)
{
    std::stringstream s;
    s << "_setup(" << rp.sys_id << "_" << rp.task_id << "_" << rp.prop_id << ")";
    s << "_rnd(" << cp.seed << "_" << cp.mns << ")";
    std::stringstream p;
    p << "_N(" << int(param(cp, "N")) << ")";
    p << "_diss(" << int(param(cp, "diss_type")) << "_" << std::setprecision(precision) << std::fixed
      << param(cp, "diss_gamma") << "_" << std::setprecision(precision) << std::fixed << param(cp, "diss_phase")
      << ")";
    p << "_drv(" << int(param(cp, "dimer_drv_type")) << "_" << std::setprecision(precision) << std::fixed
      << param(cp, "dimer_drv_ampl") << "_" << std::setprecision(precision) << std::fixed
      << param(cp, "dimer_drv_freq") << "_" << std::setprecision(precision) << std::fixed
      << param(cp, "dimer_drv_phase") << ")";
    p << "_prm(" << std::setprecision(precision) << std::fixed << param(cp, "dimer_prm_E") << "_"
      << std::setprecision(precision) << std::fixed << param(cp, "dimer_prm_U") << "_"
      << std::setprecision(precision) << std::fixed << param(cp, "dimer_prm_J") << ")";
    p << "_start(" << int(param(cp, "start_type")) << "_" << int(param(cp, "start_state")) << ")";
    return s.str() + p.str() + lpn_suffix(rp, cp) + ".txt";
}

std::string jcs_suffix(const RunParam &rp, const ConfigParam &cp, int precision)
{
    std::stringstream s;
    s << "_setup(" << rp.sys_id << "_" << rp.task_id << "_" << rp.prop_id << ")";
    s << "_rnd(" << cp.seed << "_" << cp.mns << ")";
    s << "_N(" << int(param(cp, "N")) << ")";
    s << "_diss(" << int(param(cp, "diss_type")) << "_" << std::setprecision(precision) << std::fixed
      << param(cp, "diss_gamma") << "_" << std::setprecision(precision) << std::fixed << param(cp, "diss_phase") << ")";
    s << "_drv(" << std::setprecision(precision) << std::fixed << param(cp, "jcs_drv_part_1") << "_"
      << std::setprecision(precision) << std::fixed << param(cp, "jcs_drv_part_2") << "_"
      << std::setprecision(precision) << std::fixed << param(cp, "jcs_drv_ampl") << ")";
    s << "_prm(" << std::setprecision(precision) << std::fixed << param(cp, "jcs_prm_alpha") << ")";
    s << "_start(" << int(param(cp, "start_type")) << "_" << int(param(cp, "start_state")) << ")";
    return s.str() + lpn_suffix(rp, cp) + ".txt";
}

std::string mbl_suffix(const RunParam &rp, const ConfigParam &cp, int precision)
{
    std::stringstream s;
    s << "_setup(" << rp.sys_id << "_" << rp.task_id << "_" << rp.prop_id << ")";
    s << "_rnd(" << cp.seed << "_" << cp.mns << ")";
    s << "_Nc(" << int(param(cp, "mbl_Nc")) << ")";
    s << "_rnd(" << int(param(cp, "mbl_seed")) << "_" << int(param(cp, "mbl_mns")) << ")";
    s << "_diss(" << int(param(cp, "diss_type")) << "_" << std::setprecision(precision) << std::fixed
      << param(cp, "diss_phase") << "_" << std::setprecision(precision) << std::fixed << param(cp, "diss_gamma") << ")";
    s << "_prm(" << std::setprecision(precision) << std::fixed << param(cp, "mbl_prm_W") << "_"
      << std::setprecision(precision) << std::fixed << param(cp, "mbl_prm_U") << "_"
      << std::setprecision(precision) << std::fixed << param(cp, "mbl_prm_J") << ")";
    s << "_start(" << int(param(cp, "start_type")) << "_" << int(param(cp, "start_state")) << ")";
    return s.str() + lpn_suffix(rp, cp) + ".txt";
}

std::string integrable_suffix(const RunParam &rp, const ConfigParam &cp, int precision)
{
    std::stringstream s;
    s << "_setup(" << rp.sys_id << "_" << rp.task_id << "_" << rp.prop_id << ")";
    s << "_rnd(" << cp.seed << "_" << cp.mns << ")";
    s << "_N(" << int(param(cp, "integrable_N")) << ")";
    s << "_seed(" << int(param(cp, "integrable_seed")) << ")";
    s << "_tau(" << int(param(cp, "integrable_tau")) << ")";
    s << "_k(" << int(param(cp, "integrable_k")) << ")";
    s << "_T(" << std::setprecision(precision) << std::fixed << param(cp, "integrable_T") << ")";
    return s.str() + lpn_suffix(rp, cp) + ".txt";
}

std::string ps_suffix(const RunParam &rp, const ConfigParam &cp, int precision)
{
    std::stringstream s;
    auto f = [&](const char *key) {
        std::stringstream v;
        v << std::setprecision(precision) << std::fixed << param(cp, key);
        return v.str();
    };
    s << "_setup(" << rp.sys_id << "_" << rp.task_id << "_" << rp.prop_id << ")";
    s << "_rnd(" << cp.seed << "_" << cp.mns << ")";
    s << "_s(" << int(param(cp, "ps_num_spins")) << ")";
    s << "_nps(" << int(param(cp, "ps_num_photons_states")) << ")";
    s << "_diss(" << int(param(cp, "diss_type")) << "_" << f("ps_diss_w") << ")";
    s << "_drv(" << f("ps_drv_part_1") << "_" << f("ps_drv_part_2") << "_" << f("ps_drv_ampl") << ")";
    s << "_prm(" << f("ps_prm_alpha") << "_" << f("ps_prm_d") << "_" << f("ps_prm_g") << ")";
    s << "_start(" << int(param(cp, "start_type")) << "_" << int(param(cp, "start_state")) << ")";
    return s.str() + lpn_suffix(rp, cp) + ".txt";
}

std::string dimersync_suffix(const RunParam &rp, const ConfigParam &cp, int precision)
{
    std::stringstream s;
    auto f = [&](const char *key) {
        std::stringstream v;
        v << std::setprecision(precision) << std::fixed << param(cp, key);
        return v.str();
    };
    s << "_setup(" << rp.sys_id << "_" << rp.task_id << "_" << rp.prop_id << ")";
    s << "_rnd(" << cp.seed << "_" << cp.mns << ")";
    s << "_N(" << int(param(cp, "dimersync_N")) << ")";
    s << "_diss(" << int(param(cp, "diss_type")) << "_" << f("diss_gamma") << "_" << f("diss_phase") << ")";
    s << "_drv1(" << f("dimersync_drv_ampl_1") << "_" << f("dimersync_drv_freq_1") << "_" << f("dimersync_drv_phase_1")
      << ")";
    s << "_drv2(" << f("dimersync_drv_ampl_2") << "_" << f("dimersync_drv_freq_2") << "_" << f("dimersync_drv_phase_2")
      << ")";
    s << "_T(" << int(param(cp, "dimersync_main_period")) << ")";
    s << "_prm(" << f("dimersync_prm_E") << "_" << f("dimersync_prm_U") << "_" << f("dimersync_prm_J") << ")";
    s << "_start(" << int(param(cp, "start_type")) << "_" << int(param(cp, "start_state")) << ")";
    return s.str() + lpn_suffix(rp, cp) + ".txt";
}

std::string floq2spins_suffix(const RunParam &rp, const ConfigParam &cp, int precision)
{
    std::stringstream s;
    auto f = [&](const char *key) {
        std::stringstream v;
        v << std::setprecision(precision) << std::fixed << param(cp, key);
        return v.str();
    };
    s << "_setup(" << rp.sys_id << "_" << rp.task_id << "_" << rp.prop_id << ")";
    s << "_rnd(" << cp.seed << "_" << cp.mns << ")";
    s << "_ampl(" << f("flq2sp_ampl") << ")_freq(" << f("flq2sp_freq") << ")_D1(" << f("flq2sp_Delta_1") << ")_D2("
      << f("flq2sp_Delta_2") << ")_J(" << f("flq2sp_J") << ")_gamma(" << f("flq2sp_gamma") << ")";
    return s.str() + lpn_suffix(rp, cp) + ".txt";
}

std::string floqnspins_suffix(const RunParam &rp, const ConfigParam &cp, int precision)
{
    std::stringstream s;
    auto f = [&](const char *key) {
        std::stringstream v;
        v << std::setprecision(precision) << std::fixed << param(cp, key);
        return v.str();
    };
    s << "_setup(" << rp.sys_id << "_" << rp.task_id << "_" << rp.prop_id << ")";
    s << "_rnd(" << cp.seed << "_" << cp.mns << ")";
    s << "_n(" << int(param(cp, "flqnsp_n")) << ")_ampl(" << f("flqnsp_ampl") << ")_freq(" << f("flqnsp_freq")
      << ")_D(" << f("flqnsp_Delta") << ")_J(" << f("flqnsp_J") << ")_gamma(" << f("flqnsp_gamma") << ")";
    return s.str() + lpn_suffix(rp, cp) + ".txt";
}

std::string floqspph_suffix(const RunParam &rp, const ConfigParam &cp, int precision)
{
    std::stringstream s;
    auto f = [&](const char *key) {
        std::stringstream v;
        v << std::setprecision(precision) << std::fixed << param(cp, key);
        return v.str();
    };
    s << "_setup(" << rp.sys_id << "_" << rp.task_id << "_" << rp.prop_id << ")";
    s << "_rnd(" << cp.seed << "_" << cp.mns << ")";
    s << "_nph(" << int(param(cp, "flq_sp_ph_n_ph")) << ")_ampl(" << f("flq_sp_ph_ampl") << ")_freq("
      << f("flq_sp_ph_freq") << ")_D(" << f("flq_sp_ph_Delta") << ")_O(" << f("flq_sp_ph_Omega") << ")_gamma("
      << f("flq_sp_ph_gamma") << ")";
    return s.str() + lpn_suffix(rp, cp) + ".txt";
}

std::vector<int> dump_periods(int dump_type, int dump_num, int num_obs_periods)
{
    std::vector<int> out;
    if (dump_type == 0) {
        out.assign(dump_num + 1, 0);
        const int shift = dump_num > 0 ? num_obs_periods / dump_num : 0;
        for (int i = 0; i < dump_num; i++) out[i + 1] = (i + 1) * shift;
    } else if (dump_type == 1) {
        out.assign(dump_num + 2, 0);
        const double begin_decade = std::log10(1.0);
        const double end_decade = std::log10(double(num_obs_periods));
        const double num_decades = end_decade - begin_decade;
        const double num_decades_dump = double(dump_num) / num_decades;
        for (int i = 0; i < dump_num + 1; i++) {
            const int cur = int(std::pow(10.0, begin_decade) * std::pow(10.0, (1.0 / num_decades_dump) * double(i)));
            out[i + 1] = cur > out[i] ? cur : out[i] + 1;
        }
    }
    return out;
}

static std::ofstream open_out(const std::string &fn, bool append)
{
    std::ofstream ofs(fn, append ? std::ios::app : std::ios::out);
    if (!ofs.is_open()) throw std::runtime_error("Unable to open file:\n" + fn);
    return ofs;
}

void save_double_data(const std::string &fn, const double *data, size_t n, int precision, bool append)
{
    std::ofstream ofs = open_out(fn, append);
    ofs << std::setprecision(precision) << std::scientific;
    for (size_t i = 0; i < n; i++) ofs << data[i] << std::endl;
}

void save_int_data(const std::string &fn, const int *data, size_t n, bool append)
{
    std::ofstream ofs = open_out(fn, append);
    for (size_t i = 0; i < n; i++) ofs << data[i] << std::endl;
}

void save_complex_data(const std::string &fn, const double *data, size_t n, int precision, bool append)
{
    std::ofstream ofs = open_out(fn, append);
    ofs << std::setprecision(precision) << std::scientific;
    for (size_t i = 0; i < n; i++) ofs << data[2 * i] << " " << data[2 * i + 1] << std::endl;
}

void save_2d_inv_double_data(const std::string &fn, const double *data, int rows, int cols, int precision,
                             bool append)
{
    std::ofstream ofs = open_out(fn, append);
    ofs << std::setprecision(precision) << std::scientific;
    for (int r = 0; r < rows; r++) {
        for (int c = 0; c < cols; c++) ofs << data[(size_t)c * rows + r] << " ";
        ofs << std::endl;
    }
}

void save_2d_inv_complex_data(const std::string &fn, const double *data, int rows, int cols, int precision,
                              bool append)
{
    std::ofstream ofs = open_out(fn, append);
    ofs << std::setprecision(precision) << std::scientific;
    for (int r = 0; r < rows; r++) {
        for (int c = 0; c < cols; c++) {
            const size_t i = (size_t)c * rows + r;
            ofs << data[2 * i] << " " << data[2 * i + 1] << " ";
        }
        ofs << std::endl;
    }
}

void save_2d_complex_vector(const std::string &fn, const std::vector<std::vector<std::complex<double>>> &vec,
                            int precision)
{
    std::ofstream f(fn);
    f << std::setprecision(precision) << std::scientific;
    const int dim_1 = (int)vec.size();
    const int dim_2 = dim_1 ? (int)vec[0].size() : 0;
    for (int i2 = 0; i2 < dim_2; i2++) {
        for (int i1 = 0; i1 < dim_1 - 1; i1++) f << vec[i1][i2] << "\t";
        f << vec[dim_1 - 1][i2] << std::endl;
    }
}

void save_double_vector(const std::string &fn, const std::vector<double> &v, int precision, bool append)
{
    std::ofstream ofs = open_out(fn, append);
    ofs << std::setprecision(precision) << std::scientific;
    for (double x : v) ofs << x << std::endl;
}

void save_int_vector(const std::string &fn, const std::vector<int> &v, bool append)
{
    std::ofstream ofs = open_out(fn, append);
    for (int x : v) ofs << x << std::endl;
}

// ---------------------------------------------------------------- MKL-style generators
static unsigned long long mulmod(unsigned long long a, unsigned long long b, unsigned long long m, bool pow2)
{
    if (pow2) return (a * b) & m;  // mod 2^59: m holds the mask
    return (unsigned long long)((unsigned __int128)a * b % m);
}

static unsigned long long powmod(unsigned long long a, unsigned long long e, unsigned long long m, bool pow2)
{
    unsigned long long r = 1;
    while (e) {
        if (e & 1) r = mulmod(r, a, m, pow2);
        a = mulmod(a, a, m, pow2);
        e >>= 1;
    }
    return r;
}

LeapfrogLCG LeapfrogLCG::mcg31(unsigned long long seed, unsigned long long k, unsigned long long s)
{
    const unsigned long long m = 2147483647ull, a = 1132489760ull;
    LeapfrogLCG g;
    g.m_mask_or_mod = m;
    g.pow2 = false;
    unsigned long long x0 = seed % m;
    if (x0 == 0) x0 = 1;
    g.x = mulmod(powmod(a, k + 1, m, false), x0, m, false);
    g.a_step = powmod(a, s, m, false);
    return g;
}

LeapfrogLCG LeapfrogLCG::mcg59(unsigned long long seed, unsigned long long k, unsigned long long s)
{
    const unsigned long long mask = (1ull << 59) - 1, a = 302875106592253ull;  // 13^13
    LeapfrogLCG g;
    g.m_mask_or_mod = mask;
    g.pow2 = true;
    unsigned long long x0 = seed & mask;
    if (x0 == 0) x0 = 1;
    g.x = mulmod(powmod(a, k + 1, mask, true), x0, mask, true);
    g.a_step = powmod(a, s, mask, true);
    return g;
}

double LeapfrogLCG::next()
{
    const double u = pow2 ? double(x) * 0x1p-59 : double(x) / double(m_mask_or_mod);
    x = mulmod(x, a_step, m_mask_or_mod, pow2);
    return u;
}

std::vector<double> random_observables(int d, int num, int seed, int mns, int type)
{
    const size_t dd = (size_t)d * d;
    std::vector<double> R(2 * dd * (size_t)(num > 0 ? num : 0), 0.0);
    const double two_pi = 2.0 * 3.1415926535897932384626433832795;
    std::vector<double> gr(dd), gi(dd);
    for (int o = 0; o < num; o++) {
        LeapfrogLCG st = LeapfrogLCG::mcg31(3873247ull, (unsigned long long)(seed + o), (unsigned long long)mns);
        auto gauss = [&](std::vector<double> &out) {
            for (size_t i = 0; i < out.size(); i++) {
                const double u1 = st.next(), u2 = st.next();
                out[i] = std::sqrt(-2.0 * std::log(u1)) * std::sin(two_pi * u2);
            }
        };
        gauss(gr);
        gauss(gi);
        double *r = R.data() + 2 * dd * o;
        // R = X X^H, X = 0.5 (gr + i gi)
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                double sr = 0.0, si = 0.0;
                for (int k = 0; k < d; k++) {
                    const double ar = 0.5 * gr[(size_t)i * d + k], ai = 0.5 * gi[(size_t)i * d + k];
                    const double br = 0.5 * gr[(size_t)j * d + k], bi = -0.5 * gi[(size_t)j * d + k];
                    sr += ar * br - ai * bi;
                    si += ar * bi + ai * br;
                }
                r[2 * ((size_t)i * d + j)] = sr;
                r[2 * ((size_t)i * d + j) + 1] = si;
            }
        if (type > 0) {
            double tr = 0.0;
            for (int i = 0; i < d; i++) tr += r[2 * ((size_t)i * d + i)];
            if (type == 2) tr = tr / double(d);
            for (size_t e = 0; e < 2 * dd; e++) r[e] = r[e] / tr;
        }
    }
    return R;
}

}  // namespace qjxio

#include "../../include/qjx_b200.h"

extern "C" qjx_status qjx_random_observables(int d, int num, int seed, int mns, int type, double *out)
{
    if (d < 1 || num < 0 || (num > 0 && !out) || mns < 1) return QJX_ERR_INVALID_ARG;
    const std::vector<double> R = qjxio::random_observables(d, num, seed, mns, type);
    std::copy(R.begin(), R.end(), out);
    return QJX_OK;
}
