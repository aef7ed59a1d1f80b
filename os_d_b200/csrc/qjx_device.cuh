// qjx_device.cuh -- device-side building blocks of the QJ trajectory engine (sm_100a).
//
// Arithmetic contract (bit-identical to the CPU oracle):
//   * complex matvec: per output, k ascending from 0, per k
//       re = fma(Mr, xr, re); re = fma(-Mi, xi, re); im = fma(Mr, xi, im); im = fma(Mi, xr, im)
//   * norm_square: n = n + (re*re + im*im), rows ascending, no contraction
//   * everything else literal; this translation unit is compiled with -fmad=false and the
//     intended fused operations are written as __fma_rn.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace qjx {

// ---- launch geometry of the micro-step kernel ----
constexpr int kThreads = 512;          // 16 warps (micro-step kernel)
constexpr int kNC = 32;                // trajectory columns per sub-tile (max)
constexpr int kKB = 16;                // k rows per propagator slab (8 k pairs)
constexpr int kStages = 2;             // slab pipeline depth
constexpr int kMaxGroups = 256;        // distinct matrices in one engine
constexpr int kMaxMD = 1024;           // d <= 1024 (plain form; the split form takes d <= 256)
constexpr double kSplitNormSlack = 1e-4;  // split precision: tolerated norm excess over 1
constexpr int kMaxSplitStages = 8;        // split precision: deepest operand ring
// Thread layouts of a sub-tile (rows ty + TY i, columns tx + TX j, TY * TX = 256):
//   TY = 32: MD = 32 * MT padded rows, TX = 8 column threads, up to 4 columns each
//   TY = 16: MD = 16 * MT padded rows, TX = 16 column threads, up to 2 columns each
// The host picks the layout with fewer padded rows.

// ---- trajectory phases ----
enum Phase : int {
    PH_STEP = 0,    // split step U[b][lvl] psi
    PH_REC_W = 1,   // jump-channel weight ||L_sub psi_hat||^2 g_sub
    PH_REC_A = 2,   // apply chosen channel L_sub psi_hat / sqrt(w/g)
    PH_OBS_E = 3,   // energy <psi_hat| H + E0 Hd |psi_hat>
    PH_OBS_R = 4,   // random observable sub
    PH_DONE = 5,
    PH_ERROR = 6,
    PH_RK = 7       // RK propagator: right-hand side of stage rk_stage, matrix rk_part
};

// state slots of the RK propagator (psi slots 0 and 1 hold psi and the spare copy)
constexpr int kSlotArgs = 2, kSlotK1 = 3, kSlotND = 6, kRkSlots = 7;

enum ErrCode : int { ERR_NONE = 0, ERR_NORM = 1, ERR_ZERO_W = 2, ERR_RNG = 3, ERR_TIMEOUT = 6 };

constexpr int kRecheck = -2;  // column_epilogue: the trajectory goes to the FP64 recheck list

// Per-trajectory state (one 144-byte record per trajectory).
struct __align__(16) TrajState {
    double t;          // times_all
    double eta;        // etas_all
    double ran;        // channel-choice uniform drawn at the jump (recovery's first draw)
    double tmpw;       // running sum of channel weights
    long long rng_pos; // next draw index
    unsigned long long mask;  // bit l = step counter of split level l (0 or 1)
    int lvl, b, phase, cur;   // level, branch, phase, slot holding psi
    int sub, pc, di, jumps;   // channel / observable index, periods done, next dump, jumps_counts
    int nrec, err, paused;
    int rng_src;       // trajectory whose jump stream this one draws (itself, or the base it was
                       // copied from by the Lyapunov task: vslCopyStream, experiment.cpp:2228-2256)
    // RK propagator (prop_id 1)
    double rk_h;       // step being integrated: rk_step, or the begin / end part around a jump
    double rk_prev;    // norm of psi before the step
    double rk_end;     // end part still to integrate after a located jump
    int rk_sid;        // RK: step index within the period; QJ: units done in the current branch
    int rk_stage;      // 1..4: right-hand side being evaluated
    int rk_part;       // 0: H_eff arg, 1: H_drv arg
    int rk_ctx;        // 0: step checked for a crossing; 1: begin part of a located jump
    int ens;           // ensemble of the trajectory (batched engines; 0 otherwise)
    int rechk;         // split form: this step's norm test waits for its FP64 recheck
};
static_assert(sizeof(TrajState) == 144, "TrajState layout");

struct Params {
    int d, MD, n, deep, nb, nd, nr, G;
    int gL0, gHE, gR0;
    const double2 *mats;     // [G][d][MD]  transposed matrices: mats[g][k][row]
    double2 *psi;            // [2][n][MD]
    TrajState *st;           // [n]
    double *gn;              // [n][nd] channel weights
    const double *g;         // [nd]
    const double *dt;        // [deep]
    int *cnt;                // [3][G]
    int *lists;              // [2][G][n]
    // rng
    int rng_kind;
    unsigned long long seed;
    long long tr_base;
    const double *inj_u;
    const long long *inj_off;
    // run
    int record;
    int target;
    int sub_target;  // deep tasks, qjx_run_sub_periods: stop after this many sub-periods (0: off)
    const int *dump_at;
    int n_dumps;
    int dump_base;
    // observables
    int keep_adr;
    double *o_norm, *o_mean, *o_disp, *o_m2, *o_energy;  // [max_dumps][n]
    double2 *o_robs;                                        // [max_dumps][n][nr]
    double *o_adr;                                          // keep_adr ? [max_dumps][n][d] : [n][d]
    double *mean_start;                                     // [n]
    // jump records, record-major [rec_cap][n]
    int rec_cap;
    double *r_time, *r_norm, *r_eta;
    int *r_type;
    // control: [0] error count, [1] first error trajectory, [2] paused count, [3] first error code,
    //          [4] timeouts
    int *ctrl;
    long long *work;         // [0] trajectory-matvecs executed
    // optional per-CTA trace, accumulated over micro-steps: [grid][kTraceFields] clock64 cycles
    // and counts (null: tracing off)
    long long *trace;
    // split-precision form: bf16 hi/lo planes of Re M and Im M of every matrix in tcgen05
    // core-matrix order
    int split;                    // 0 FP64 plain form, 1 split bf16x3
    int MDs, KS;                  // rows padded to 16 (MMA N), k-steps of 16 complex components
    int sstages;                  // depth of the split kernel's operand ring
    const unsigned char *usplit;  // [G][KS][4 planes: Re hi, Re lo, Im hi, Im lo][MDs rows x 16 k] bf16
    // per ensemble: rows padded to 16 (MMA N) and k-steps; per group: byte offset of its B planes
    // in usplit
    const int *e_mds, *e_ks;
    const long long *g_uoff;
    // tile plan of the next micro-step: [0] rows per tile, [1 + g] first tile of group g,
    // [1 + G] tiles in all; written by the last CTA of a micro-step (or split_plan_kernel)
    int *splan;
    int grid;                     // CTAs of the micro-step kernels
    // near-threshold FP64 rechecks of the split form: band (relative to the norm; 0: off), the
    // recheck lists of the micro-steps ([3] counts, [2][n] trajectories) and the k rows of the
    // FP64 matrix slabs streamed through the operand ring
    double recheck_tol;
    int *rcnt;
    int *rlist;
    int rchk_kb;
    int min_rows;                 // split form: fewest trajectories per tcgen05 tile (tile shape)
    // RK propagator (prop 1): groups 0 and 1 are H_eff and H_drv; psi has kRkSlots slots
    int prop;                     // 0 QJ split tree, 1 RK
    int rk_ns, period0, drv_type;
    double rk_step, T, E0, A, drv_freq, drv_phase;
    // deep tasks (StdDeep): each branch runs brep = 2 deep_num_steps units of two level-0 steps;
    // with subdump the observables are taken after every sub-period (two units)
    int brep, subdump;
    // run_periods advances trajectories [0, n_active) only (the Lyapunov task's transient runs
    // the bases alone), and of those only the ones with active[tr] != 0 when `active` is set
    // (the ensemble slots of a serving engine)
    int n_active;
    const unsigned char *active;
    // plain step kernel tiling, per ensemble (chosen from its padded rows and the shared memory):
    // columns per sub-tile (32, 16 or 8) and k rows per propagator slab; step_smem is the
    // kernel's dynamic shared memory (the largest ensemble layout)
    const int *e_nc, *e_kb;
    int step_smem;
    // ensembles (a batched engine holds E ensembles of their own dimension, operators, seed and
    // period; an ordinary engine is the batch of one).  Trajectories [e_tr0[e], e_tr0[e+1]) form
    // ensemble e; its groups are e_g0[e] + the local group (branch * deep + level, gL0 + channel,
    // gHE, gR0 + observable).  d and MD above are the largest dimension and its padded rows.
    int E;
    const int *e_d;                   // [E] dimension
    const int *e_tr0;                 // [E + 1] first trajectory
    const int *e_g0;                  // [E] first group
    const double *e_dt;               // [E][nb][deep] split-level steps
    const double *e_rate;             // [E][nd] jump rates
    const unsigned long long *e_seed; // [E] Philox key
    const long long *e_sbase;         // [E] Philox stream of the ensemble's first trajectory
    const long long *g_off;           // [G] offset of the group's matrix in mats (double2 units)
    const int *g_ens;                 // [G] ensemble of the group
    const long long *g_loff;          // [G] start of the group's bucket list (capacity: the
                                      // ensemble's trajectories); lists hold 2 x ltot entries
    long long ltot;
    // plain step kernel plan of the next micro-step: [0, G] bucket starts, [G + 1, 2G + 1] cost
    // prefix; written by the last CTA of a micro-step (or plan_kernel after a host call)
    int *plan;
    unsigned int *plan_sync;          // [1] CTAs finished in the current micro-step
    unsigned int *gen;                // [1] split form: plans made (the grid barrier of a multi-step launch)
    int *sdone;                       // [1] split form: micro-steps run since the host last cleared it
};

// Dimension, split-level steps and jump rates of a trajectory's ensemble.
__device__ __forceinline__ int dim_of(const Params &P, const TrajState &s) { return P.e_d[s.ens]; }
__device__ __forceinline__ const double *dt_of(const Params &P, const TrajState &s)
{
    return P.e_dt + ((size_t)s.ens * P.nb + s.b) * P.deep;
}
__device__ __forceinline__ double rate_of(const Params &P, const TrajState &s, int i)
{
    return P.e_rate[(size_t)s.ens * P.nd + i];
}

// Lyapunov paired trajectories (task_id 7, LpnMult): [0, n/2) bases, n/2 + b the variation of b.
struct LpnParams {
    int lpn_type;        // -1 mean, -2 energy, k >= 0 random observable k
    int eps_deep;        // bisection halvings at most
    int per_period;      // lambda_per_periods
    double eps_low, eps_high, eps_error, delta_s, delta_f_high, delta_f_low, max_energy;
    double *lambda, *lambda_now, *delta_s_v, *mean_lpn, *energy_lpn;  // [n]
    double2 *robs_lpn;                                                // [n][nr]
    int *num_renorms;                                                 // [n]
    long long *var_pos;                                               // [n] variation-stream draws
    int *renormed;                                                    // [n] last call
    double *ratio, *ds_rec, *df_rec;                                  // [n] last call
    int *eps_iters;                                                   // [n] last bisection
    double *eps;                                                      // [n] last bisection
    const int *pair0;                                                 // [E + 1] first pair of each ensemble
    int pairs;                                                        // sum over ensembles of n_e / 2
    int mbl_Nc;                                                       // > 0: MBL characteristics
    int chars_sys;                                                    // characteristics of sys_id 0 / 1 / 3 / 5
    double spec_div;                                                  // MBL: spec = robs slot 0 / W
    const int *words;                                                 // MBL: [d] basis words
};
// trace fields: total, setup (bucket scan + gather), operand wait, MMA loop, epilogue,
// sub-tiles, 8-column blocks, columns
constexpr int kTraceFields = 8;

// ---------------------------------------------------------------- Philox4x32-10
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
        const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// Uniform in (0,1]: draw `idx` of trajectory `tr` (identical to the host definition).
__device__ __forceinline__ double philox_uniform(unsigned long long seed, unsigned long long tr,
                                                 unsigned long long idx)
{
    const unsigned long long blk = idx >> 1;
    uint32_t c[4] = {(uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)tr, (uint32_t)(tr >> 32)};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint32_t a = (idx & 1) ? c[2] : c[0];
    const uint32_t b = (idx & 1) ? c[3] : c[1];
    const unsigned long long m = ((unsigned long long)(a >> 5) << 26) | (unsigned long long)(b >> 6);
    return __dmul_rn((double)(m + 1), 0x1p-53);
}

// Next uniform of a trajectory; sets *err on an exhausted injected sequence.  The Philox
// stream of local trajectory i of ensemble e is e_sbase[e] + i under the key e_seed[e], so an
// ensemble draws the same numbers alone and inside a batch.
__device__ __forceinline__ double draw(const Params &P, int tr, TrajState &s, int *err)
{
    (void)tr;
    if (P.rng_kind == 0)
        return philox_uniform(P.e_seed[s.ens], (unsigned long long)(P.e_sbase[s.ens] + (s.rng_src - P.e_tr0[s.ens])),
                              (unsigned long long)(s.rng_pos++));
    const long long lo = P.inj_off[s.rng_src], hi = P.inj_off[s.rng_src + 1];
    if (lo + s.rng_pos >= hi) { *err = ERR_RNG; return 0.5; }
    return P.inj_u[lo + (s.rng_pos++)];
}

// ---------------------------------------------------------------- canonical reductions
// Lane l holds the literal running sum of the terms with index l, l+32, ... (ascending);
// the 32 partial sums are combined by an xor butterfly over offsets 16, 8, 4, 2, 1.  IEEE
// addition is commutative, so every lane ends with the same value, and the CPU oracle
// reproduces it exactly.
__device__ __forceinline__ double warp_allsum(double s)
{
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, off));
    return s;
}

__device__ __forceinline__ double warp_norm(const double2 *x, int d, int lane)
{
    double s = 0.0;
    for (int i = lane; i < d; i += 32) {
        const double2 v = x[i];
        s = __dadd_rn(s, __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y)));
    }
    return warp_allsum(s);
}

// ---------------------------------------------------------------- TMA bulk copies + mbarriers
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: gives up after `limit` polls and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, long long limit)
{
    for (long long i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 1-D TMA bulk copy global -> shared, completion counted in bytes on `bar`.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace qjx
