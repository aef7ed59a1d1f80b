/*
 * qjx_oracle.h -- CPU restatement of the QJX quantum-jump path (TEST INFRASTRUCTURE).
 *
 * This library is the oracle the CUDA engine in os_d_b200 is tested against.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.  The product
 * never links or calls it.
 *
 * It restates, in plain C, the reference's algorithm for sys_id 0 (Bose dimer),
 * task_id 1 (Std), prop_id 0 (QJ):
 *   operators          source/cpp/QJX/QJX/newdel.cpp:3-37, 450-498, 1454-1498, 2285-2388
 *   split tree / expm  source/cpp/QJX/QJX/qj_proc.cpp:4-120, core.cpp:9880-9926
 *   period bisection   source/cpp/QJX/QJX/qj_proc.cpp:264-343, core.cpp:84-95
 *   norm test / jump   source/cpp/QJX/QJX/experiment.cpp:1239-1382
 *   observables        source/cpp/QJX/QJX/core.cpp:665-725, experiment.cpp:1395-1469, 2023-2078
 *   Std task flow      source/cpp/QJX/QJX/experiment.cpp:411-542, 3249-3271
 *   dump schedule      source/cpp/QJX/QJX/newdel_exp.cpp:408-455
 *
 * Parity status: the reference needs Intel MKL and Eigen, neither of which exists in
 * this image, and it ships no golden data, so this restatement is "parity unpinned"
 * against the reference binary.  It is pinned instead to independent known-answer
 * tests (closed-form operators, scipy expm, Philox KAT vectors, dense Lindblad).
 *
 * Arithmetic contract (shared bit-for-bit with the CUDA engine):
 *   complex matvec out_i = sum_k M_ik x_k, k ascending from 0, per k:
 *       re = fma(Mr, xr, re); re = fma(-Mi, xi, re); im = fma(Mr, xi, im); im = fma(Mi, xr, im)
 *   reductions over the d components (norm_square, mean, m2, energy, random observables):
 *       32 lane sums, lane l = literal running sum over i = l, l+32, ... ascending, then an
 *       xor butterfly over offsets 16, 8, 4, 2, 1 (a GPU warp's shfl_xor reduction)
 *   every other expression is evaluated literally (compiled with -ffp-contract=off).
 *
 * Complex arrays are interleaved (re, im) doubles, matrices row-major d x d, like
 * MKL_Complex16 in the reference.
 */
#ifndef QJX_ORACLE_H
#define QJX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Dimer operators (newdel.cpp).  Outputs are complex d x d, d = N + 1:
 *   H   : hamiltonian            (newdel.cpp:450-498)
 *   Hd  : hamiltonian_drv        (newdel.cpp:485)
 *   L   : dissipators[0]         (newdel.cpp:1454-1498)
 *   K0,K1: hamiltonians_qj[0/1] = -i (H - i/2 gamma L^H L + E_b Hd), gamma = g/N,
 *          E_0 = E + A, E_1 = E - A  (newdel.cpp:2285-2388) */
int orc_dimer_operators(int N, double J, double U, double E, double A, double g,
                        double *H, double *Hd, double *L, double *K0, double *K1);

/* JCS operators (sys_id 1, newdel.cpp:96-130, 564-649, 1546-1580, 2499-2601): d = N; H, H_drv,
 * L = a, the number operator Nop = a^+ a, K0 = -i H_eff + E0 H_drv, K1 = -i H_eff, all complex d x d. */
int orc_jcs_operators(int N, double alpha, double drv_ampl, double *H, double *Hd, double *L, double *Nop,
                      double *K0, double *K1);

/* MBL (sys_id 3, newdel.cpp:182-271, 868-958, 1699-1815, 2751-2838).  orc_mbl_basis: the words with
 * Nc/2 of Nc bits set, ascending (returns their number d = C(Nc, Nc/2); id_to_x may be NULL).
 * orc_mbl_operators: energies[Nc], H, L [num_diss][d][d] (num_diss = Nc for diss_type 0, Nc - 1 for
 * diss_type 1), K = hamiltonians_qj[0]; jump rates are 1.  orc_mbl_imbalance: get_imbalance_mbl
 * (experiment.cpp:1753-1800) of n adr rows [n][d]. */
int orc_mbl_basis(int Nc, int *id_to_x);
void orc_mcg31_uniform(unsigned long long seed, unsigned long long k, unsigned long long s, int count, double a,
                       double b, double *out);
int orc_mbl_operators(int Nc, double W, double U, double J, int mbl_seed, int mbl_mns, int diss_type, double diss_phase,
                      double gamma, double *energies, double *H, double *L, double *K);
void orc_mbl_imbalance(int Nc, int d, int n, const double *adr, double *out);

/* PS (sys_id 2, newdel.cpp:132-181, 650-866, 1582-1697, 2603-2749): d = 2^ns nps; H, Hd, L [1 (+ ns)],
 * S [4] = special, special_2, special_3, special_4, K0 (kick), K1, all complex d x d. */
int orc_ps_operators(int ns, int nps, double alpha, double dprm, double gprm, double drv_ampl, int diss_type,
                     double diss_w, double *H, double *Hd, double *L, double *S, double *K0, double *K1);

/* Integrable (sys_id 5, newdel.cpp:310-345, 1030-1095, 1924-2076, 2914-3004): d = 2^N, H = 0, L [N][d][d]
 * (the con 4 x 4 on neighbouring spins and on the border pair), special (the spec observable), K. */
int orc_integrable_operators(int N, int seed, int num_seeds, double tau, double kk, double *L, double *special,
                             double *K);

/* Floq2Spins (sys_id 7, newdel.cpp:346-378, 1096-1182, 2077-2136, 3005-3101): d = 4; H (= special),
 * L [2], K = hamiltonians_qj[0] (undriven). */
int orc_floq2spins_operators(double D1, double D2, double J, double gamma, double *H, double *L, double *K);

/* FloqManySpins (sys_id 8, newdel.cpp:379-413, 1184-1332, 2138-2224, 3103-3199): d = 2^n; H (= special),
 * L [n], K = hamiltonians_qj[0] (undriven). */
int orc_floqnspins_operators(int n, double Delta, double J, double gamma, double *H, double *L, double *K);

/* FloqSpinPh (sys_id 9, newdel.cpp:414-449, 1334-1452, 2226-2284, 3201-3297): d = 2 (n_ph + 1); H (= special),
 * L = a (x) 1, K = hamiltonians_qj[0] (undriven). */
int orc_floqspph_operators(int n_ph, double Delta, double Omega, double gamma, double *H, double *L, double *K);

/* H_eff = H - (i/2) gamma L^H L, gamma = g / N (newdel.cpp:2293-2352): the non_drv_part of the RK
 * propagator (newdel.cpp:2354-2366), complex d x d. */
int orc_dimer_heff(int N, double J, double U, double E, double g, double *Heff);

/* Matrix exponential exp(A), complex n x n, Higham (2005) scaling and squaring with
 * Pade [m/m], m in {3,5,7,9,13}.  Replaces Eigen MatrixXcd::exp() (qj_proc.cpp:55,98). */
int orc_expm(int n, const double *A, double *out);

/* Split tree of one branch: U_l = exp(K * dt_l), dt_l = T * 2^-(l+2), l = 0..deep-1,
 * dt computed by repeated halving like init_split_branches (qj_proc.cpp:15-24). */
int orc_split_tree(int d, const double *K, double T, int deep, double *U_out);

/* Philox4x32-10 (Salmon et al., SC'11).  ctr[4], key[2] -> out[4]. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Uniform in (0,1]: draw number `idx` of trajectory `tr` under `seed`. */
double orc_philox_uniform(uint64_t seed, uint64_t tr, uint64_t idx);

/* One ensemble problem for the QJ engine. */
typedef struct {
    int d;              /* sys_size = N + 1 */
    int n_traj;
    int deep;           /* ex_deep */
    int num_branches;   /* num_ham_qj (2 for the dimer) */
    int num_diss;       /* 1 for the dimer */
    int num_robs;       /* random observables */
    int record;         /* params "jump": 0 none, 1 times+types, 2 also norms+etas */
    int rng_kind;       /* 0 = Philox(seed, tr, idx); 1 = injected per-trajectory uniforms */
    double T;           /* period */
    uint64_t seed;
    const double *U;    /* [num_branches][deep][d][d] complex */
    const double *L;    /* [num_diss][d][d] complex */
    const double *g;    /* [num_diss] rates (1.0 for the dimer) */
    const double *HE;   /* [d][d] complex: H + E0 * Hd (energy observable) */
    const double *R;    /* [num_robs][d][d] complex random observables */
    const double *inj_u;      /* rng_kind 1: concatenated uniforms */
    const int64_t *inj_off;   /* rng_kind 1: [n_traj + 1] offsets into inj_u */
    uint64_t tr_base;         /* Philox stream of local trajectory tr is tr_base + tr (sharding) */
    const double *branch_len; /* [num_branches] branch durations (NULL: T / 2 each, the dimer's
                                 half periods); level l of branch b steps 2 len_b 2^-(l+2) */
} orc_problem;

/* Mutable per-run state and outputs. */
typedef struct {
    double *phi;        /* [n_traj][d] complex, current states (in/out) */
    double *eta;        /* [n_traj] */
    double *t;          /* [n_traj] times_all */
    int64_t *rng_pos;   /* [n_traj] next draw index */
    int *jumps_counts;  /* [n_traj] */
    int64_t *matvecs;   /* [n_traj] complex matvecs executed (work counter) */
    /* jump records, capacity cap per trajectory; n_rec[tr] = records written */
    int rec_cap;
    int *n_rec;
    double *jump_times; /* [n_traj][rec_cap] */
    double *jump_norms;
    double *jump_etas;
    int *diss_types;
    int *error;         /* [n_traj] 0 ok; 1 norm>1; 2 all jump weights zero; 3 rng exhausted; 4 record overflow */
    int *rng_src;       /* [n_traj] jump stream each trajectory draws from (NULL: its own) */
} orc_state;

/* Initial state: start_type 0 -> |start_state>, else uniform sqrt(1/d) (newdel_exp.cpp:656-679);
 * draw eta_0 (experiment.cpp:3260-3265).  Sets t = 0, counts = 0. */
int orc_init(const orc_problem *p, orc_state *s, int start_type, int start_state);

/* Advance trajectories [tr0, tr1) by n_periods periods; is_obs gates jump recording
 * exactly like ed->is_obs (qj_proc.cpp:296).  OpenMP over trajectories. */
int orc_run_periods(const orc_problem *p, orc_state *s, int tr0, int tr1, int n_periods, int is_obs, int n_threads);

/* Deep tasks (task_id 4, StdDeep): n_units runs of branch b from split level 0; a sub-period is
 * two units (one_sub_period_deep, qj_proc.cpp:345-359; ex_period_obs_deep, core.cpp:114-153).
 * The problem's T must be the tree head's dt, T_period / (2 deep_num_steps). */
int orc_run_branch_units(const orc_problem *p, orc_state *s, int tr0, int tr1, int b, int n_units, int is_obs,
                         int n_threads);

/* RK propagator (prop_id 1): dpsi/dt = -i (H_eff + E(t) H_drv) psi by classic RK4 with rk_ns
 * steps per period and a jump located by linear interpolation of the norm inside a step.
 *   rk_period          source/cpp/QJX/QJX/core.cpp:439-450 (t = period T + step rk_step)
 *   rk_step_dimer      core.cpp:11886-11948 (crossing, begin / end parts, recursion)
 *   rk_int_dimer       core.cpp:11592-11619; rk_right_part_dimer core.cpp:11033-11115
 *   arg_upd / rk_final / rk_recovery / save / restore   rk_proc.cpp:124-341 (arg_upd always
 *                      uses the full rk_step, also inside begin and end parts)
 * ND = non_drv_part (H_eff), DR = drv_part (H_drv) (newdel.cpp:2354-2366). */
typedef struct {
    const double *ND;   /* [d][d] complex */
    const double *DR;   /* [d][d] complex */
    double E0, A, freq, phase;
    int drv_type;       /* 1: E0 + A sin(freq t + phase); otherwise E0 +/- A on the half periods */
    int rk_ns;          /* steps per period */
} orc_rk;

/* Advance trajectories [tr0, tr1) by n_periods periods with the RK propagator; the periods are
 * numbered period0, period0 + 1, ... (the reference's period_id). */
int orc_run_periods_rk(const orc_problem *p, const orc_rk *rk, orc_state *s, int tr0, int tr1, int n_periods,
                       int period0, int is_obs, int n_threads);

/* Observables of every trajectory (calc_chars_std[_start], core.cpp:665-725).
 * mean_start is written when is_start != 0 and read otherwise.  adr may be NULL. */
int orc_observables(const orc_problem *p, const orc_state *s, int is_start,
                    double *mean_start, double *norm, double *mean, double *dispersion,
                    double *m2, double *energy, double *robs /* [n_traj][num_robs] complex */,
                    double *adr /* [n_traj][d] */);

/* Dump schedule (newdel_exp.cpp:408-455).  Returns dump_num_total, fills periods
 * (caller provides dump_num + 2 ints). */
int orc_dump_periods(int dump_type, int dump_num, int num_obs_periods, int *periods);

/* Lyapunov paired trajectories (task_id 7, LpnMult; lpn_oracle.c).  n_traj is even; [0, n/2) are the
 * bases and n/2 + b the variation of base b.  s->rng_src must be set (a variation draws the jump
 * stream of its base after every copy). */
typedef struct {
    int lpn_type;        /* -1 mean, -2 energy, k >= 0 random observable k */
    int eps_deep;        /* lpn_eps_deep: bisection halvings at most */
    int per_period;      /* lambda_per_periods: 0 renormalise on the thresholds, 1 every period */
    int pad;
    double eps_low, eps_high, eps_error;  /* log10 bounds of eps, tolerance on delta_s */
    double delta_s;      /* lpn_delta_s */
    double delta_f_high, delta_f_low;
    double max_energy;   /* max |Re H_ii| (lpn_type -2) */
    /* MBL characteristics (MBLCoreBehaviour, core.cpp:4729-4902) when mbl_Nc > 0: random-observable
     * slot 0 holds H and spec = slot 0 / spec_div (W); mean = the imbalance of the adr row;
     * lpn_type -1 = |spec_b - spec_v|, -2 = |imbalance_v - imbalance_b|, k >= 0 = slot k + 1.
     * chars_sys selects the system: 0 the dimer, 1 JCS (JCSCoreBehaviour, core.cpp:2739-2975: slot 0
     * holds a, spec = slot 0 / alpha, mean_lpn = <a^+ a> (the energy observable), -1 = |spec_b -
     * spec_v|, -2 = |n_v - n_b| / d), 3 MBL (with mbl_Nc), 5 Integrable (core.cpp:6470-6676: slot 0
     * holds the special matrix, spec_div 1, -1 = |spec_b - spec_v|, no -2). */
    int mbl_Nc;
    int chars_sys;
    double spec_div;
} orc_lpn_config;

typedef struct {
    double *lambda, *lambda_now, *delta_s;   /* [n_traj] */
    double *mean_lpn, *energy_lpn;            /* [n_traj] */
    double *robs_lpn;                         /* [n_traj][num_robs] complex */
    int *num_renorms;                         /* [n_traj] */
    int64_t *var_pos;                         /* [n_traj] draws taken from the variation stream */
    /* last call: renormalised?, delta_f / delta_s, delta_s, delta_f (save_lambdas records) */
    int *renormed;
    double *ratio, *ds_rec, *df_rec;
    int *eps_iters;                           /* halvings of the last bisection */
    double *eps;                              /* eps of the last bisection */
} orc_lpn;

/* After the bases' transient periods: copy every base into its variation (phi, eta, jump stream),
 * perturb it (var_trajectory_lpn) and set the Lyapunov characteristics (calc_chars_lpn_start). */
int orc_lpn_start(const orc_problem *p, orc_state *s, const orc_lpn_config *cfg, orc_lpn *lp);
/* After one observation period: calc_chars_lpn of the bases and lambda_lpn (per_period 0) or
 * lambda_lpn_now (1) of the variations, curr_time = (period_id + 1) T. */
int orc_lpn_period(const orc_problem *p, orc_state *s, const orc_lpn_config *cfg, orc_lpn *lp, double curr_time);
/* calc_chars_lpn of the bases only (LpnMultDeep sub-periods without a Lyapunov step). */
int orc_lpn_bases(const orc_problem *p, orc_state *s, const orc_lpn_config *cfg, orc_lpn *lp);
/* pow(10, x) and log(x) of the Lyapunov task, shared operation for operation with the engine. */
double orc_lpn_exp10(double x);
double orc_lpn_log(double x);

/* Canonical kernels, exported for unit tests. */
void orc_matvec(int d, const double *M, const double *x, double *out);
double orc_norm_square(int d, const double *x);
/* Ensemble purity Tr(rho^2), rho = (1/n) sum_tr psi_hat psi_hat^dagger (psi [n][d] complex
 * interleaved); the formula of calc_purity (source/cpp/CQdiss/CQdiss/CalcTraseRO2.cpp:57-75).
 * rho (d x d complex, may be NULL) receives the matrix. */
double orc_purity(int d, int n, const double *psi, double *rho);

#ifdef __cplusplus
}
#endif
#endif
