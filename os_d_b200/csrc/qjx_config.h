// qjx_config.h -- the reference's parameter-file interface and output writers (host C++).
//
// config.txt: typed "key value" lines, only lines that split (on single spaces, empty
// tokens dropped) into exactly two tokens are used (source/cpp/QJX/QJX/config.cpp:3-27,
// 101-117); unknown keys are ignored.  params.txt: "key double" lines into a string ->
// double map (config.cpp:124-142).  Defaults follow RunParam / ConfigParam
// (source/cpp/QJX/QJX/config.h:60-139).
#pragma once
#include <complex>
#include <map>
#include <string>
#include <vector>

namespace qjxio {

struct RunParam {
    int sys_id = 0, task_id = 0, prop_id = 0;
    int is_debug = 0, is_pp = 0;
    std::string init_fn, path;
    int num_threads = 1;
};

struct ConfigParam {
    std::map<std::string, double> params;
    std::string fn_suffix;
    int num_tp_periods = 0, num_obs_periods = 10, num_trajectories = 1;
    int seed = 0, mns = 1000000;
    int ex_deep = 16, rk_ns = 1000;
};

// Splits on the delimiter, dropping empty tokens (config.cpp:3-27).
std::vector<std::string> split(const std::string &str, const std::string &delim);
void set_param(RunParam &rp, ConfigParam &cp, const std::string &key, const std::string &val);
// Returns false when a file could not be opened (the reference then keeps the defaults).
bool read_config(RunParam &rp, ConfigParam &cp, const std::string &fn_config);
bool read_params(ConfigParam &cp, const std::string &fn_params);
// The "#### parameters ####" echo of output_params (config.cpp:147-181).
std::string params_echo(const RunParam &rp, const ConfigParam &cp);

// Value of a params.txt key; throws std::runtime_error naming a missing key (the reference
// dereferences find() unchecked).
double param(const ConfigParam &cp, const std::string &key);
double param_or(const ConfigParam &cp, const std::string &key, double dflt);

// DimerOutputBehavior::suffix_param with precision 4 (source/cpp/QJX/QJX/outputter.cpp:3-44,
// 353-388): _setup(s_t_p)_rnd(seed_mns)_N(..)_diss(..)_drv(..)_prm(..)_start(..).txt
std::string dimer_suffix(const RunParam &rp, const ConfigParam &cp, int precision = 4);
// JCSOutputBehavior::suffix_param (source/cpp/QJX/QJX/outputter.cpp:95-133)
std::string jcs_suffix(const RunParam &rp, const ConfigParam &cp, int precision = 4);
// MBLOutputBehavior::suffix_param (source/cpp/QJX/QJX/outputter.cpp:176-212)
std::string mbl_suffix(const RunParam &rp, const ConfigParam &cp, int precision = 4);
// IntegrableOutputBehavior::suffix_param (source/cpp/QJX/QJX/outputter.cpp:244-269)
std::string integrable_suffix(const RunParam &rp, const ConfigParam &cp, int precision = 4);
// PSOutputBehavior::suffix_param (source/cpp/QJX/QJX/outputter.cpp:135-174)
std::string ps_suffix(const RunParam &rp, const ConfigParam &cp, int precision = 4);
// DimerSyncOutputBehavior::suffix_param (source/cpp/QJX/QJX/outputter.cpp:45-93)
std::string dimersync_suffix(const RunParam &rp, const ConfigParam &cp, int precision = 4);
// Floq2SpinsOutputBehavior::suffix_param (source/cpp/QJX/QJX/outputter.cpp:271-299)
std::string floq2spins_suffix(const RunParam &rp, const ConfigParam &cp, int precision = 4);
// FloqManySpinsOutputBehavior::suffix_param (source/cpp/QJX/QJX/outputter.cpp:299-326)
std::string floqnspins_suffix(const RunParam &rp, const ConfigParam &cp, int precision = 4);
// FloqSpinPhOutputBehavior::suffix_param (source/cpp/QJX/QJX/outputter.cpp:326-353)
std::string floqspph_suffix(const RunParam &rp, const ConfigParam &cp, int precision = 4);

// init_dump_periods (source/cpp/QJX/QJX/newdel_exp.cpp:408-455); empty on a bad dump_type.
std::vector<int> dump_periods(int dump_type, int dump_num, int num_obs_periods);

// Writers with the reference's formats (source/cpp/QJX/QJX/utils.cpp, utils.h):
// setprecision(precision) << scientific, one value per line, "re im" pairs, rows x cols with a
// trailing space, complex values as "(re,im)" separated by tabs.
void save_double_data(const std::string &fn, const double *data, size_t n, int precision, bool append);
void save_int_data(const std::string &fn, const int *data, size_t n, bool append);
void save_complex_data(const std::string &fn, const double *data, size_t n, int precision, bool append);
// complex data[col * rows + row] (interleaved re, im) printed as rows lines of "re im " pairs
// (save_2d_inv_complex_data, utils.cpp:228-282, the non-append branch)
void save_2d_inv_complex_data(const std::string &fn, const double *data, int rows, int cols, int precision,
                              bool append);
// data[col * rows + row] printed as rows lines of cols values (save_2d_inv_double_data)
void save_2d_inv_double_data(const std::string &fn, const double *data, int rows, int cols, int precision,
                             bool append);
// vec[col][row] complex printed as rows lines, columns separated by '\t' (save_2d_vector)
void save_2d_complex_vector(const std::string &fn, const std::vector<std::vector<std::complex<double>>> &vec,
                            int precision);
void save_double_vector(const std::string &fn, const std::vector<double> &v, int precision, bool append);
void save_int_vector(const std::string &fn, const std::vector<int> &v, bool append);

// MKL VSL basic generators restated from their published definitions (Intel MKL Vector
// Statistics notes): MCG31m1 x_n = 1132489760 x_{n-1} mod (2^31 - 1); MCG59
// x_n = 13^13 x_{n-1} mod 2^59; u_n = x_n / m; a leapfrog stream (k, s) yields x_{k+1+i*s}.
// Box-Muller (VSL_RNG_METHOD_GAUSSIAN_BOXMULLER): x = sqrt(-2 ln u1) sin(2 pi u2).
// No MKL exists in this image, so agreement with MKL's streams is unverified.
struct LeapfrogLCG {
    unsigned long long m_mask_or_mod, a_step, x;
    bool pow2;
    static LeapfrogLCG mcg31(unsigned long long seed, unsigned long long k, unsigned long long s);
    static LeapfrogLCG mcg59(unsigned long long seed, unsigned long long k, unsigned long long s);
    double next();
};
// Random observable matrices of init_random_obs (source/cpp/QJX/QJX/newdel.cpp:3652-3750):
// X = 0.5 (G_re + i G_im), R = X X^H, scaled by 1/tr (type 1) or d/tr (type 2).
std::vector<double> random_observables(int d, int num, int seed, int mns, int type);

}  // namespace qjxio
