/*
 * qjx_b200.h -- C ABI of the B200 quantum-jump trajectory engine (os_d_b200).
 *
 * Plain pointers and sizes only; no exceptions cross this boundary; every call returns
 * a qjx_status and qjx_last_error() gives the message.  Complex arrays are interleaved
 * (re, im) doubles, matrices row-major d x d, exactly like MKL_Complex16 arrays in the
 * reference (source/cpp/QJX/QJX/data.h:36-58).  The caller owns every host buffer; the
 * engine owns its device memory and copies in/out.  A handle is bound to one CUDA
 * stream and is not re-entrant; distinct handles may run concurrently.
 *
 * Which reference interface each entry point replaces:
 *   qjx_create           init_split_structure_dimer + copies per thread
 *                        (source/cpp/QJX/QJX/core.cpp:6-22, 9880-9926; qj_proc.cpp:122-167)
 *   qjx_set_states       StdNewDelBehaviour::init_data -> init_basic_data / init_start_state
 *                        (source/cpp/QJX/QJX/newdel_exp.cpp:98-117, 332-375, 656-679)
 *   qjx_set_uniforms     the per-trajectory VSL streams (newdel_exp.cpp:244-296): the caller
 *                        may inject any pre-generated uniform sequence instead of Philox
 *   qjx_init_thresholds  eta_0 draw of trans_process_single (experiment.cpp:3249-3265)
 *   qjx_run_periods      the OpenMP loop over trajectories calling PropagateBehavior::one_period
 *                        -> DimerCoreBehaviour::ex_period -> one_period_branch
 *                        (experiment.cpp:411-430, 477-501; propagator.cpp:27-30; core.cpp:84-95;
 *                        qj_proc.cpp:271-343), batched over all trajectories, with the
 *                        per-dump calc_chars_std fused in (core.cpp:697-725)
 *   qjx_reset_times      resresh_times (experiment.cpp:2214-2219)
 *   qjx_observe          calc_chars_std_start / calc_chars_std (core.cpp:665-725)
 *   qjx_get_observables  ed->norm_evo / mean_evo / ... arrays (core.cpp:795-816)
 *   qjx_get_jumps        ed->jump_times / diss_types / jump_norms / jump_etas (qj_proc.cpp:296-307,
 *                        experiment.cpp:1371-1374)
 *   qjx_build_dimer      DimerNewDelBehaviour::init_sizes/init_hamiltonians/init_dissipators/
 *                        init_hamiltonians_qj + init_split_branches (newdel.cpp:3-37, 450-498,
 *                        1454-1498, 2285-2388; qj_proc.cpp:4-120)
 *   qjx_fb_*             f-basis Lindblad RK4 (source/cpp/CQdiss_os_dimer/CQdiss/calcODE.cpp:75-118,
 *                        249-389)
 */
#ifndef QJX_B200_H
#define QJX_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    QJX_OK = 0,
    QJX_ERR_INVALID_ARG = 1,
    QJX_ERR_OOM = 2,
    QJX_ERR_NORM_GT_ONE = 3,        /* replaces the throw in is_norm_crossed (experiment.cpp:1247-1251) */
    QJX_ERR_RNG_EXHAUSTED = 4,      /* injected uniform sequence of a trajectory ran out */
    QJX_ERR_ZERO_JUMP_WEIGHTS = 5,  /* every jump channel had zero weight (reference loops forever) */
    QJX_ERR_TIMEOUT = 6,            /* a bounded device wait gave up */
    QJX_ERR_CUDA = 7,
    QJX_ERR_UNSUPPORTED = 8,
    QJX_ERR_STATE = 9
} qjx_status;

typedef struct qjx_engine qjx_engine;

/* Tile shapes of the micro-step kernels.  All zero: the engine's rule, or the choice the autotuner
 * (qjx_autotune) cached for this dimension and precision.  Tiles never change results: every
 * output keeps its own summation order whatever the tiling. */
typedef struct {
    int nc;      /* plain form: trajectory columns per sub-tile (32, 16 or 8) */
    int kb;      /* plain form: k rows per propagator slab (even, 2..16) */
    int stages;  /* split form: depth of the operand ring (2..8) */
    int rows;    /* split form: fewest trajectories per tcgen05 tile (multiple of 8, 8..128) */
} qjx_tiles;

typedef struct {
    int d;             /* sys_size (N + 1 for the dimer) */
    int n_traj;        /* num_trajectories */
    int deep;          /* ex_deep: split levels per branch */
    int num_branches;  /* num_ham_qj */
    int num_diss;      /* number of jump operators */
    int num_robs;      /* number of random observables */
    double T;          /* period */
    int record;        /* params "jump": 0 none, 1 times + types, 2 also norms + etas */
    int rng_kind;      /* 0: Philox4x32-10 (seed, trajectory, draw index); 1: injected uniforms */
    uint64_t seed;
    int rec_cap;       /* jump records buffered on the device per trajectory (0 -> 1024) */
    int keep_adr;      /* 0: keep the latest |psi_k|^2/|psi|^2 only; 1: keep it for every dump */
    int max_dumps;     /* capacity of the observable arrays (dump_num_total) */
    int device;        /* CUDA device ordinal */
    int64_t tr_base;   /* global index of trajectory 0 (Philox stream id = tr_base + local index), so
                          an ensemble sharded over GPUs draws exactly the numbers of one big run */
    int deep_num_steps; /* 0: Std task.  > 0: StdDeep task (task_id 4): every branch runs as
                          2 deep_num_steps units of the split tree of T_sub = T / (2 deep_num_steps)
                          (give U from qjx_build_dimer_deep), and observation runs (is_obs 1) take
                          the observables after every sub-period into consecutive dump slots from
                          dump_base, num_branches deep_num_steps per period (ex_period_obs_deep,
                          core.cpp:114-153); dump_at must then be empty. */
    int precision;     /* 0: complex FP64 end to end (the reference's arithmetic, bit-exact with the
                          oracle); 1: split precision: every d x d matvec runs on the tcgen05 tensor
                          cores as bf16 hi/lo planes with FP32 accumulation (products hi*hi + hi*lo +
                          lo*hi), states, norms, thresholds, jump times and renormalisation stay
                          FP64.  Needs d <= 256.  QJX has no such mode
                          (its zgemv is FP64).  A split engine runs a batch of micro-steps as one
                          cooperative launch (one CTA per SM); when another context holds SMs it
                          runs them one launch each, with the same results ($QJX_SPLIT_COOP=0
                          selects that from the start). */
    const double *branch_len; /* [num_branches] durations of the branches of a period (NULL: T / 2
                          each, the dimer's half periods); systems with unequal parts (the JCS kick
                          and free evolution, init_split_structure_jcs, core.cpp:10086-10124) give
                          them here.  Level l of branch b steps 2 len_b / brep 2^-(l+2), brep = 1
                          or 2 deep_num_steps. */
    double split_recheck; /* split form (precision 1): a norm test whose split-precision norm p lies
                          within split_recheck * p of the threshold is not decided; that step's
                          matvec is computed again in FP64 (the plain form's arithmetic) in the next
                          micro-step and decides.  0 selects 1e-5 (about 5x the measured split error
                          of the norm), a negative value turns the recheck off. */
    qjx_tiles tiles;   /* tile shapes (all 0: rule or autotuner cache) */
} qjx_config;

typedef struct {
    int64_t micro_steps;     /* lock-step micro-steps launched */
    int64_t matvecs;         /* complex d x d matvecs executed (trajectory-steps) */
    int64_t jumps;           /* jumps recorded */
    double kernel_ms;        /* device time of run/observe calls, first to last launch (CUDA events) */
    double last_call_ms;     /* device time of the last run/observe call */
    double step_kernel_ms;   /* device time of the micro-step kernel batches alone (CUDA events) */
    int64_t launches;        /* kernels launched by the engine */
    int64_t mma_tiles;       /* split form: 128-row tcgen05 tiles (12 MMAs of 128 x MDs x 16 per k-step) */
    int64_t rechecks;        /* split form: norm tests taken again on an FP64 matvec */
} qjx_stats;

/* U: [num_branches][deep][d][d] split propagators exp(K_b dt_l), dt_l = T 2^-(l+2).
 * L: [num_diss][d][d] jump operators; g: [num_diss] rates (head->g, core.cpp:9905).
 * HE: [d][d] energy operator H + E0 * H_drv (experiment.cpp:1440).  R: [num_robs][d][d]. */
qjx_status qjx_create(const qjx_config *cfg, const double *U, const double *L, const double *g,
                      const double *HE, const double *R, qjx_engine **out);
/* The RK propagator (prop_id 1): RKPropagateBehavior::one_period -> rk_period / rk_step_dimer
 * (source/cpp/QJX/QJX/propagator.cpp:67-129, core.cpp:439-450, 11033-11115, 11592-11619,
 * 11886-11948, rk_proc.cpp:124-341): classic RK4 of dpsi/dt = -i (H_eff + E(t) H_drv) psi with
 * rk_ns steps per period, E(t) = E0 +/- A on the half periods (drv_type 0) or
 * E0 + A sin(drv_freq t + drv_phase) (drv_type 1), the jump time located by linear
 * interpolation of the norm inside the crossing step.  H_eff = non_drv_part, H_drv = drv_part
 * (newdel.cpp:2354-2366).  cfg's deep / num_branches are ignored; precision must be 0.  Periods
 * are numbered from the last qjx_reset_times (or creation), like the reference's period_id. */
qjx_status qjx_create_rk(const qjx_config *cfg, const double *H_eff, const double *H_drv, double E0, double A,
                         int drv_type, double drv_freq, double drv_phase, int rk_ns, const double *L,
                         const double *g, const double *HE, const double *R, qjx_engine **out);
/* One ensemble of a batched engine: its own dimension, trajectories, period, Philox key and first
 * stream (the thresholds it would draw in an engine of its own with seed = seed and
 * tr_base = tr_base), and its operators with the layouts of qjx_create at this d. */
typedef struct {
    int d;
    int n_traj;
    double T;
    uint64_t seed;
    int64_t tr_base;
    const double *U, *L, *g, *HE, *R;
} qjx_ensemble;
/* Batched engine: n_ens ensembles of uneven Hilbert dimension (d <= 1024) advanced together by
 * the same persistent micro-step launches (every (ensemble, matrix) pair is a bucket of the
 * grouped GEMM; a sub-tile multiplies only its ensemble's d x d block).  cfg supplies what the
 * ensembles share: deep, num_branches, num_diss, num_robs, record, rng_kind, rec_cap, keep_adr,
 * max_dumps, device, deep_num_steps, precision (1 needs every ensemble's d <= 256; each then has
 * its own bf16 planes, k-steps and padded rows); cfg's d, n_traj, T, seed and tr_base are
 * ignored.  Trajectories are numbered ensemble after ensemble; states and
 * observables use the largest dimension as row length (qjx_set_states: rows zero-padded past
 * each ensemble's d).  Every trajectory is bit-identical to its run in an engine of its own.
 * The Lyapunov entry points, qjx_purity and the RK propagator take single-ensemble engines. */
qjx_status qjx_create_batch(const qjx_config *cfg, int n_ens, const qjx_ensemble *ens, qjx_engine **out);
/* Serving engine: n_slots resident ensemble slots, each with room for dimension <= d_cap and
 * n_cap trajectories (slot s owns trajectories s * n_cap ...); all slots start free.  Run calls
 * advance the loaded slots together (qjx_create_batch's launches); loading or releasing a slot
 * between run calls leaves the others' states, streams and records untouched, so requests join
 * and leave a running batch (continuous batching).  cfg as for qjx_create_batch. */
qjx_status qjx_create_slots(const qjx_config *cfg, int n_slots, int d_cap, int n_cap, qjx_engine **out);
/* Load an ensemble into a free slot: its operators into the slot's resident matrix region, its
 * e->n_traj trajectories from psi ([n_traj][e->d] complex; NULL: |0>), fresh times, records and
 * thresholds (its own Philox stream), then the slot runs with the next run call. */
qjx_status qjx_slot_load(qjx_engine *h, int slot, const qjx_ensemble *e, const double *psi);
/* Stop advancing and observing a slot; its states stay readable until it is loaded again. */
qjx_status qjx_slot_release(qjx_engine *h, int slot);
/* Free and total device memory of `device` in bytes (cudaMemGetInfo), for admission by footprint. */
qjx_status qjx_mem_info(int device, size_t *free_bytes, size_t *total_bytes);
/* Device bytes an engine holds (all its allocations). */
qjx_status qjx_engine_bytes(qjx_engine *h, size_t *bytes);
void qjx_destroy(qjx_engine *h);
const char *qjx_last_error(const qjx_engine *h);
const char *qjx_status_string(qjx_status s);

/* psi: [n_traj][d] complex initial states; resets times, counters and records. */
qjx_status qjx_set_states(qjx_engine *h, const double *psi);
/* Injected uniforms (rng_kind 1): u concatenated, offsets [n_traj + 1]. */
qjx_status qjx_set_uniforms(qjx_engine *h, const double *u, const int64_t *offsets);
qjx_status qjx_init_thresholds(qjx_engine *h);
/* Advance every trajectory by n_periods periods.  is_obs gates jump recording like ed->is_obs.
 * dump_at[i] (ascending, 1..n_periods) are period counts, relative to this call, after which
 * observables are taken into dump slot dump_base + i. */
qjx_status qjx_run_periods(qjx_engine *h, int n_periods, int is_obs, const int *dump_at, int n_dumps,
                           int dump_base);
qjx_status qjx_reset_times(qjx_engine *h);
/* Deep tasks (deep_num_steps > 0, QJ propagator): continue every active trajectory for n_sub
 * sub-periods from where the previous call left it, the observables after each sub-period going to
 * dump slots dump_base, dump_base + 1, ... (LpnMultDeep runs the Lyapunov update between
 * sub-periods: ex_period_obs_deep_mult_lpn, core.cpp:155-241).  Periods carry over between calls;
 * qjx_run_periods always starts a new period. */
qjx_status qjx_run_sub_periods(qjx_engine *h, int n_sub, int dump_base);
/* Observables of the current states into dump slot `dump`; is_start writes mean_start. */
qjx_status qjx_observe(qjx_engine *h, int dump, int is_start);
/* Per-dump arrays laid out [dump][trajectory]; robs [dump][trajectory][num_robs] complex;
 * adr [dump][trajectory][d] (keep_adr 1) or [trajectory][d] latest (keep_adr 0).  NULL skips. */
qjx_status qjx_get_observables(qjx_engine *h, int dump0, int n_dumps, double *norm, double *mean,
                               double *dispersion, double *m2, double *energy, double *robs, double *adr);
qjx_status qjx_get_mean_start(qjx_engine *h, double *mean_start);
/* Ensemble purity Tr(rho^2) of the current states, rho = (1/n_traj) sum |psi_hat><psi_hat|
 * with psi_hat = psi/||psi||.  QJX has no ensemble purity; the formula is calc_purity's
 * (source/cpp/CQdiss/CQdiss/CalcTraseRO2.cpp:57-75) for the density matrix the trajectories
 * sample.  rho (optional, NULL skips) receives the d x d matrix row-major, complex interleaved.
 * Sharded ensembles combine rho_total = sum_r n_r rho_r / sum_r n_r before squaring. */
qjx_status qjx_purity(qjx_engine *h, double *purity, double *rho);
/* Current states [n_traj][d] complex, times, etas, jump counts (any pointer may be NULL). */
qjx_status qjx_get_states(qjx_engine *h, double *psi, double *t, double *eta, int *jumps_counts);
/* Jump records of one trajectory accumulated since qjx_set_states. */
qjx_status qjx_jump_count(qjx_engine *h, int tr, int64_t *count);
qjx_status qjx_get_jumps(qjx_engine *h, int tr, double *times, int *types, double *norms, double *etas);
qjx_status qjx_get_stats(qjx_engine *h, qjx_stats *stats);

/* The project's tile autotuner (no counterpart in the reference, which has no tiles): times the
 * candidate tile shapes of cfg->precision (plain: sub-tile columns x slab rows; split: ring depth x
 * fewest rows per tile) on scratch engines of cfg with the given operators (cfg->n_traj
 * trajectories from |0>, one untimed period, then n_periods timed periods of device time) and
 * returns the fastest in *best.  cand / us (capacity *n_cand; NULL to skip) receive every
 * candidate and its device microseconds per trajectory-period; *n_cand the count.  The winner is
 * stored under (precision, d) in the tile cache file: $QJX_TILE_CACHE, else
 * $HOME/.cache/qjx_b200/tiles.txt; engines created later with all-zero cfg->tiles use it. */
qjx_status qjx_autotune(const qjx_config *cfg, const double *U, const double *L, const double *g, const double *HE,
                        int n_periods, qjx_tiles *best, qjx_tiles *cand, double *us, int *n_cand);
/* Later qjx_run_periods calls advance trajectories [0, n_active) only (the others keep their
 * states); the Lyapunov task runs its transient on the bases alone (LpnMultExperimentBehaviour::
 * trans_process, experiment.cpp:147-155).  n_active = n_traj restores the default. */
qjx_status qjx_set_active(qjx_engine *h, int n_active);

/* Lyapunov paired trajectories (task_id 7, LpnMult; experiment.cpp:138-286).  n_traj is even;
 * trajectories [0, n/2) are the bases and n/2 + b is the variation of base b -- in a batched engine
 * within every ensemble (each with an even n_traj), so a whole parameter sweep runs as one batch.
 * qjx_set_bases_only(h, 1): later run calls advance the bases of every ensemble only (the
 * transient); 0 restores all. */
qjx_status qjx_set_bases_only(qjx_engine *h, int on);
typedef struct {
    int lpn_type;         /* -1 mean, -2 energy, k >= 0 random observable k (calc_delta_s, core.cpp:839-901) */
    int eps_deep;         /* lpn_eps_deep: bisection halvings at most */
    int per_period;       /* lambda_per_periods: 0 lambda_lpn (renormalise on the thresholds), 1
                             lambda_lpn_now (every period) */
    int pad;
    double eps_low, eps_high;  /* lpn_eps_low / lpn_eps_high: log10 bounds of the perturbation size */
    double eps_error;     /* lpn_eps_error: tolerance on delta_s */
    double delta_s;       /* lpn_delta_s: target distance after a perturbation */
    double delta_f_high, delta_f_low;  /* lpn_delta_f_high / lpn_delta_f_low */
    double max_energy;    /* max |Re H_ii| of the hamiltonian (init_obs_lpn, newdel_exp.cpp:540-550) */
    /* Whose Lyapunov characteristics (chars_sys = the reference's sys_id; 0: the dimer's).
     * 3 MBL (MBLCoreBehaviour, core.cpp:4729-4902) with mbl_Nc (every ensemble has d =
     * C(mbl_Nc, mbl_Nc/2); 0 otherwise): random-observable slot 0 holds H, spec = slot 0 / spec_div
     * (W), mean_lpn is the imbalance, lpn_type -1 = |spec_b - spec_v|, -2 = |imbalance_v -
     * imbalance_b|.  1 JCS (JCSCoreBehaviour, core.cpp:2739-2975): slot 0 holds a, spec = slot 0 /
     * spec_div (alpha), mean_lpn is <a^+ a> (the energy observable with Nop), -1 = |spec_b - spec_v|,
     * -2 = |n_v - n_b| / d.  5 Integrable (IntegrableCoreBehaviour, core.cpp:6470-6676): slot 0 holds
     * the special matrix, spec_div 1, -1 = |spec_b - spec_v|, no -2.  For all three, k >= 0 = random
     * observable slot k + 1. */
    int mbl_Nc;
    int chars_sys;
    double spec_div;
} qjx_lpn_config;
/* After the bases' transient (trans_process, experiment.cpp:138-183): copy every base into its
 * variation (psi, eta and jump stream: copy_trajectory_lpn, experiment.cpp:2221-2244), perturb
 * it (var_trajectory_lpn, experiment.cpp:2278-2397; the direction is drawn from a per-trajectory
 * variation stream) and set the Lyapunov characteristics (calc_chars_lpn_start, core.cpp:727-761).
 * Follow with qjx_reset_times and qjx_observe(h, 0, 1). */
qjx_status qjx_lpn_start(qjx_engine *h, const qjx_lpn_config *cfg);
/* After one observation period (obser_process, experiment.cpp:209-240): calc_chars_lpn of the
 * bases and lambda_lpn / lambda_lpn_now of the variations with curr_time = (period_id + 1) T.
 * adr_dump >= 0: this period carried dump slot adr_dump, whose |psi_i|^2/|psi|^2 of the variations
 * is replaced by the value after the update (abs_diag_rho_all after lambda_lpn); -1 otherwise. */
qjx_status qjx_lpn_period(qjx_engine *h, double curr_time, int adr_dump);
/* LpnMultDeep (task_id 8): calc_chars_lpn of the bases only, for the sub-periods at which the
 * variations take no Lyapunov step (lambda_per_periods 1: ex_period_obs_deep_mult_lpn,
 * core.cpp:155-241, updates them at the last sub-period of a period only). */
qjx_status qjx_lpn_bases(qjx_engine *h);
/* Current Lyapunov values per trajectory [n_traj] (robs_lpn [n_traj][num_robs] complex); any
 * pointer may be NULL.  lambda_now is what lambda / lambda_evo dump (core.cpp:959-1000). */
qjx_status qjx_lpn_get(qjx_engine *h, double *lambda_now, double *lambda, double *delta_s, double *mean_lpn,
                       double *energy_lpn, double *robs_lpn, int *num_renorms);
/* Renormalisations of the last qjx_lpn_start / qjx_lpn_period per trajectory: renormed (0/1),
 * delta_f / delta_s, delta_s, delta_f (the save_lambdas records, experiment.cpp:3082-3088), the
 * bisection halvings and the perturbation size eps; any pointer may be NULL. */
qjx_status qjx_lpn_get_last(qjx_engine *h, int *renormed, double *ratio, double *delta_s, double *delta_f,
                            int *eps_iters, double *eps);
/* Checkpoint / resume (preemption): the complete trajectory state between run calls -- every
 * state slot, the per-trajectory records (times, thresholds, RNG cursors, branch / level,
 * jump counters), channel weights, mean_start, the period counter and, when started, the
 * Lyapunov arrays -- as one host blob.  Loading it into an engine created with the same
 * configuration continues the run bit for bit (jump records already drained to the host are
 * not part of the blob).  QJX has no checkpoint (its only resume is skipping finished jobs). */
qjx_status qjx_checkpoint_size(qjx_engine *h, size_t *bytes);
qjx_status qjx_checkpoint_save(qjx_engine *h, void *buf, size_t bytes);
qjx_status qjx_checkpoint_load(qjx_engine *h, const void *buf, size_t bytes);
/* Per-CTA trace of the micro-step kernel (profiling aid, off by default): enabling clears
 * and starts accumulating, per persistent CTA, clock64 cycles {total, setup, (reserved),
 * MMA loop, epilogue} and counts {sub-tiles, 8-column blocks, columns}.  qjx_get_trace
 * copies [n_ctas][n_fields] int64 (out may be NULL to query the shape). */
qjx_status qjx_set_trace(qjx_engine *h, int enable);
qjx_status qjx_get_trace(qjx_engine *h, int64_t *out, int *n_ctas, int *n_fields);
/* Measured FP64 throughput of the device in TFLOP/s (2 flops per FMA): an FFMA-chain
 * microbenchmark and an m8n8k4 FP64 tensor-core (DMMA) chain microbenchmark; the larger is
 * the roofline peak of the FP64 contraction.  Either pointer may be NULL. */
qjx_status qjx_measure_fp64_peak(int device, double *ffma_tflops, double *dmma_tflops);

/* Dimer model on the host (FP64): H, Hd, L [d][d]; K [2][d][d] = hamiltonians_qj
 * -i (H - i/2 (g/N) L^H L + (E +- A) Hd); Utree [2][deep][d][d] = exp(K_b T 2^-(l+2)),
 * T = 2 pi / omega.  Any output may be NULL. */
qjx_status qjx_build_dimer(int N, double J, double U, double E, double A, double g, double omega, int deep,
                           double *H, double *Hd, double *L, double *K, double *Utree);
/* A split tree built on the GPU (for serving; no counterpart in the reference, which exponentiates
 * every level on the host, QJX/qj_proc.cpp:55,98): for nb generators K_b (complex [d][d] row-major,
 * e.g. qjx_build_dimer's K), Utree [nb][deep][d][d] = exp(K_b head_b 2^-(l+2)).  The finest level is a
 * degree-14 Taylor series of K dt / 2^s with 1-norm at most 1/4, squared s times; every coarser level
 * is the square of the next finer (the tree's dt halves per level).  FP64 complex GEMMs on `device`
 * on a private stream (stream-ordered allocations, no device-wide synchronisation); agrees with the
 * host build to about 1e-12. */
qjx_status qjx_expm_tree(int d, int nb, const double *K, const double *head, int deep, int device, double *Utree);
/* The JCS system (sys_id 1; newdel.cpp:96-130, 564-649, 1546-1580, 2499-2601; split structure
 * core.cpp:10086-10157): d = N, H = 0.5/alpha^3 a^+a^+aa, H_drv = a^+ - a, L = a, the number
 * operator Nop = a^+ a and the observable `special` A_op = a; K_0 = -i H_eff + E0 H_drv (the kick),
 * K_1 = -i H_eff with gamma = 1/(4 alpha); Utree [2][deep][d][d] = exp(K_b head_b 2^-(l+2)) with
 * head_b = part_b alpha.  A period runs each part as two halves (the head's two children): engine
 * branches [U_0, U_0, U_1, U_1] with qjx_config.branch_len [head_0, head_0, head_1, head_1] / 2.
 * Any output pointer may be NULL. */
qjx_status qjx_build_jcs(int N, double alpha, double drv_ampl, double part_1, double part_2, int deep, double *H,
                         double *Hd, double *L, double *Nop, double *A_op, double *Kout, double *Utree);
/* The MBL system (sys_id 3; MBLNewDelBehaviour, newdel.cpp:182-271, 868-958, 1699-1815, 2751-2838):
 * Nc cells (even, <= 24) holding Nc/2 hard-core particles, basis = the Nc-bit words with Nc/2 bits
 * set in ascending order (id_to_x [d], d = C(Nc, Nc/2)); energies [Nc] = uniform(-1, 1) disorder
 * from the MCG31 stream seed 77778888 leapfrogged (mbl_seed, mbl_mns); H = W sum_c n_c e_c +
 * U sum_c n_c n_{c+1} - J (nearest-neighbour hops); L [num_diss][d][d]: diss_type 0 n_c (num_diss
 * = Nc), diss_type 1 n_c - n_{c+1} plus the hop c <-> c+1 with phase diss_phase (num_diss = Nc - 1);
 * K = -i (H - i/2 gamma sum_c L_c^H L_c); jump rates 1.  Utree [deep][d][d] = exp(K T 2^-(l+2)):
 * one branch, run twice per period of duration T (init_split_structure_mbl, core.cpp:10382-10432).
 * Any output pointer may be NULL (Utree also skips the exponentials). */
qjx_status qjx_mbl_size(int Nc, int diss_type, int *d, int *num_diss);
qjx_status qjx_build_mbl(int Nc, double W, double U, double J, int mbl_seed, int mbl_mns, int diss_type,
                         double diss_phase, double gamma, double T, int deep, double *energies, int *id_to_x,
                         double *H, double *L, double *K, double *Utree);
/* The PS system (sys_id 2; PSNewDelBehaviour, newdel.cpp:132-181, 650-866, 1582-1697, 2603-2749): ns
 * spins times nps photon states, d = 2^ns nps (spins (x) photons, spin 0 the most significant);
 * H = (d_prm/2) J_z + (g_prm/2)(J_- a^+ + J_+ a) + 0.5/alpha^3 a^+a^+aa, H_drv = a^+ - a; L [1 + ns
 * for diss_type 1]: a, then sigma_- of each spin; S [4][d][d] = a, J_z, J_+, a^+a (spec, spec_2,
 * spec_3, photons); K [2] = -i H_eff + E0 H_drv (the kick), -i H_eff with gamma 1/(4 alpha) on the
 * cavity and diss_w on the spins; jump rates 1; Utree [2][deep][d][d] = exp(K_b head_b 2^-(l+2)),
 * head_b = part_b alpha, each part run as two halves (init_split_structure_ps, core.cpp:10234-10305:
 * engine branches [K_0, K_0, K_1, K_1] of durations head_b / 2).  Any output pointer may be NULL. */
qjx_status qjx_build_ps(int ns, int nps, double alpha, double d_prm, double g_prm, double drv_ampl, int diss_type,
                        double diss_w, double part_1, double part_2, int deep, double *H, double *Hd, double *L,
                        double *S, double *K, double *Utree);
/* The Integrable system (sys_id 5; IntegrableNewDelBehaviour, newdel.cpp:310-345, 1030-1095, 1924-2076,
 * 2914-3004): N spins (3 <= N <= 10), d = 2^N, H = 0; L [N][d][d]: the 4 x 4 operator tau |00><00| +
 * k |11><11| + |01><10| + |10><01| on spins (c, c+1), c < N - 1, and on the border pair (N-1, 0);
 * special = y / sqrt(Re tr y^2) / sqrt(d), y = (X + X^H) / 2, X_ij = g_ij (1 + i) with g Box-Muller
 * normals of the MCG31 stream seed 13371337 leapfrogged (seed, num_seeds); K = -i (-(i/2) sum_c
 * L_c^H L_c); jump rates 1; Utree [deep][d][d] = exp(K T 2^-(l+2)), one branch run twice per period
 * (init_split_structure_integrable, core.cpp:10610-10660).  Any output pointer may be NULL. */
qjx_status qjx_build_integrable(int N, int seed, int num_seeds, double tau, double k, double T, int deep, double *L,
                                double *special, double *K, double *Utree);
/* The Floquet two-spin system (sys_id 7; Floq2SpinsNewDelBehaviour, newdel.cpp:346-378, 1096-1182,
 * 2077-2136, 3005-3101), QJ branch: d = 4, H = (Delta_1 sz (x) 1 + Delta_2 1 (x) sz)/2 + J sy (x) sy
 * (also the spec observable), L [2] = sigma_- on each spin, K = -i (H - (i/2) gamma sum L^H L), jump
 * rates 1; Utree [deep][4][4] = exp(K T 2^-(l+2)) for one branch that covers T / 2 per period
 * (init_split_structure_floq2spins, core.cpp:10722-10766); the drive enters the RK propagator only.
 * Any output pointer may be NULL. */
qjx_status qjx_build_floq2spins(double D1, double D2, double J, double gamma, double T, int deep, double *H,
                                double *L, double *K, double *Utree);
/* The Floquet many-spin system (sys_id 8; FloqManySpinsNewDelBehaviour, newdel.cpp:379-413, 1184-1332,
 * 2138-2224, 3103-3199), QJ branch: n spins (1 <= n <= 10), d = 2^n, H = (Delta / 2) sum sz + J sy^(x)n
 * (n >= 2; (Delta / 2) sz for n = 1), also the spec observable; L [n] = sigma_- on each spin; K = -i (H
 * - (i/2) gamma sum L^H L), jump rates 1; Utree [deep][d][d] = exp(K T 2^-(l+2)) for one branch covering
 * T / 2 per period (init_split_structure_floqnspins, core.cpp:10825-10871).  Any output may be NULL. */
qjx_status qjx_build_floqnspins(int n, double Delta, double J, double gamma, double T, int deep, double *H, double *L,
                                double *K, double *Utree);
/* The Floquet spin-photon system (sys_id 9; FloqSpinPhNewDelBehaviour, newdel.cpp:414-449, 1334-1452,
 * 2226-2284, 3201-3297), QJ branch: photons (x) spin (index 2 k + s), d = 2 (n_ph + 1), H = (Delta / 2)
 * sz + (Omega / 2)(a^+ sm + a sp) (also the spec observable), L [1] = a (x) 1, K = -i (H - (i/2) gamma
 * L^H L), jump rate 1; Utree [deep][d][d] for one branch covering T / 2 per period
 * (init_split_structure_flq_sp_ph, core.cpp:10928-10974).  Any output pointer may be NULL. */
qjx_status qjx_build_floqspph(int n_ph, double Delta, double Omega, double gamma, double T, int deep, double *H,
                              double *L, double *K, double *Utree);
/* The MBL imbalance of n probability rows adr [n][d] (get_imbalance_mbl, experiment.cpp:1753-1800). */
qjx_status qjx_mbl_imbalance(int Nc, int n, const double *adr, double *out);
/* qjx_build_dimer with the split tree of the deep tasks' sub-period T / (2 deep_num_steps)
 * (init_split_structure_dimer_deep, core.cpp:9928-9981). */
qjx_status qjx_build_dimer_deep(int N, double J, double U, double E, double A, double g, double omega, int deep,
                                int deep_num_steps, double *H, double *Hd, double *L, double *K, double *Utree);
/* Operators of the RK propagator: H_eff = H - (i/2)(g/N) L^H L (non_drv_part) and H_drv
 * (drv_part), built by DimerNewDelBehaviour::init_hamiltonians_qj (newdel.cpp:2285-2366). */
qjx_status qjx_build_dimer_rk(int N, double J, double U, double E, double g, double *H_eff, double *H_drv);
/* exp(A) of a complex n x n matrix, Higham (2005) scaling and squaring. */
qjx_status qjx_expm(int n, const double *A, double *out);
/* Random observables of init_random_obs (source/cpp/QJX/QJX/newdel.cpp:3652-3750): for
 * o < num, Gaussians from an MCG31m1 leapfrog stream (seed 3873247, index seed + o, stride
 * mns) with Box-Muller, X = (G_re + i G_im) / 2, R = X X^H divided by its trace (type 1) or
 * trace / d (type 2).  out: [num][d][d] complex.  The generator restates MKL's published
 * MCG31m1 / Box-Muller definitions; MKL itself is not available to confirm the stream. */
qjx_status qjx_random_observables(int d, int num, int seed, int mns, int type, double *out);

/* ---- f-basis Lindblad RK4 (density-matrix oracle of the ensemble) ---- */
typedef struct qjx_fb qjx_fb;
/* f-basis Liouvillian of the dimer (Gs, Qs_drv in CSR with sorted columns, Ks), the matrices the
 * reference assembles from structure constants (source/cpp/CQdiss_os_dimer/CQdiss/CalcQs.cpp:141-173,
 * CalcRs.cpp:385-468, CalcKs.cpp:82-135, CalcGs.cpp:3-11) for the f-basis operators of InitH.cpp:227-342
 * and Init_a1_a2.cpp:54-122 with gamma = g / N (data.cpp:11).  Call with null arrays to get the
 * nonzero counts, then with arrays of those sizes (row pointers n + 1, n = (N+1)^2 - 1). */
qjx_status qjx_fb_build_dimer(int N, double J, double U, double E, double g, int *gs_nnz, int *qs_nnz,
                              int *gs_rowptr, int *gs_col, double *gs_val, int *qs_rowptr, int *qs_col,
                              double *qs_val, double *Ks);
/* CSR (0-based) Gs and Qs_drv of size n x n, Ks [n]; x0 [n] initial f-vector.
 * drv_type 0: E(t) = -A sign(sin(w t + phase)), 1: -A sin(w t + phase) (calcODE.cpp:91-117). */
qjx_status qjx_fb_create(int n, const int *gs_rowptr, const int *gs_col, const double *gs_val,
                         const int *qs_rowptr, const int *qs_col, const double *qs_val, const double *Ks,
                         const double *x0, double drv_ampl, double drv_freq, double drv_phase, int drv_type,
                         double T, int num_steps, int device, qjx_fb **out);
/* Integrate n_periods periods of num_steps RK4 steps starting at period index period0.
 * When the system fits, one thread-block cluster (<= 16 CTAs) holds it in distributed shared
 * memory and runs a period per launch; otherwise one launch per RK stage. */
qjx_status qjx_fb_run(qjx_fb *h, int period0, int n_periods);
/* Cluster size of the cluster-resident path (0: per-stage kernels). */
qjx_status qjx_fb_info(qjx_fb *h, int *cluster_size);
qjx_status qjx_fb_get(qjx_fb *h, double *x, double *last_period_ms);
void qjx_fb_destroy(qjx_fb *h);

/* Allocation-free f-basis RK4 (no counterpart in the reference, which always runs on the host).
 * For callers that must not allocate GPU memory themselves or through this library: a host
 * program that owns every device buffer through its own pool, or a solver called from a loop
 * that must not pay cudaMalloc/cudaFree's device-wide synchronisation or fail under memory
 * pressure in the middle of a run.  Same arithmetic as qjx_fb_create + qjx_fb_run (the same
 * kernels); every pointer is DEVICE memory owned by the caller: the CSR arrays of Gs and
 * Qs_drv (0-based), Ks [n], and x [n], advanced in place by n_periods periods of num_steps RK4
 * steps starting at period index period0, four kernel launches per RK4 step.  The RK4 stage
 * vectors (two stage arguments and k1..k3) live in a static device array sized for
 * n <= QJX_FB_NOALLOC_MAX_N (2.5 MiB, held by every GPU that loads the library until the process
 * exits); larger n is rejected with QJX_ERR_UNSUPPORTED.  The return status covers this call's own
 * launches only; an earlier error of other code is neither reported nor cleared.  Work is queued on `stream`
 * (a cudaStream_t, NULL for the default stream) and the call returns without waiting.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before any stream capture.  All calls on a device
 * share the one array and it keeps the last call's contents (every element a call reads it
 * writes first, so nothing needs clearing); calls that overlap on the GPU race, so serialise
 * them on one stream per device. */
#define QJX_FB_NOALLOC_MAX_N 65536
qjx_status qjx_fb_rk4_noalloc(int n, const int *gs_rowptr, const int *gs_col, const double *gs_val,
                              const int *qs_rowptr, const int *qs_col, const double *qs_val, const double *Ks,
                              double *x, double drv_ampl, double drv_freq, double drv_phase, int drv_type, double T,
                              int num_steps, int period0, int n_periods, int device, void *stream);

#ifdef __cplusplus
}
#endif
#endif
