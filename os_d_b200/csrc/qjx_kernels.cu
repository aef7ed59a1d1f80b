// qjx_kernels.cu -- sm_100a kernels of the QJ trajectory engine.
//
// The reference advances one trajectory at a time through a recursive bisection over
// split levels (qj_proc.cpp:271-343): every step is one dense complex matvec with the
// propagator U[b][level] of its branch and level, followed by a norm test against the
// trajectory's threshold.  Jumps are frequent (about 50 per period at N = 100 and 110 at
// N = 200), so the bisection, not the jump-free stroboscopic step, is the hot path.
//
// B200 design: all trajectories advance in lock-step micro-steps.  In each micro-step
// every active trajectory needs exactly one matvec with one of G matrices (2 x ex_deep
// propagators, the jump operators, the energy operator, the random observables).  The
// trajectories are bucketed by matrix, and one persistent kernel per micro-step runs a
// grouped FP64 GEMM over the buckets:
//   * a tile is one matrix x 32 trajectory columns, full height (all d rows), so the
//     column norm needed by the jump test stays inside the CTA;
//   * the gathered state columns and the propagator K-slabs are moved by the TMA engine
//     (cp.async.bulk + mbarrier, 2-stage slab pipeline of 16 k-rows), so the tensor pipe is
//     fed while the next slab streams from L2;
//   * the epilogue is the whole trajectory state machine: norm test, descend / accept,
//     jump record, renormalisation, channel choice, threshold redraw, time bookkeeping,
//     period and dump accounting, the observables, and re-bucketing for the next step.
// FP64 has no tcgen05 kind, so the plain form's contraction runs on the FP64 tensor core
// (mma.sync m8n8k4 f64), laid out so that every output keeps the oracle's k-ascending fma
// chain (bit-identical results).  The split-precision form (qjx_split.cuh, included at the
// end) runs the same micro-steps with bf16x3 products on the tcgen05 tensor cores.
#include <algorithm>

#include "qjx_device.cuh"

namespace qjx {

constexpr long long kWaitLimit = 1ll << 24;  // bounded mbarrier polls before giving up

__device__ __forceinline__ double2 *slot_ptr(const Params &P, int slot, int tr)
{
    return P.psi + ((size_t)slot * P.n + tr) * P.MD;
}

// Whether run calls advance trajectory tr.
__device__ __forceinline__ bool runs(const Params &P, int tr)
{
    return tr < P.n_active && (!P.active || P.active[tr]);
}

// Bucket (global group) of a trajectory's next matvec, or -1.
__device__ __forceinline__ int group_of(const Params &P, const TrajState &s)
{
    int g;
    switch (s.phase) {
    case PH_STEP: g = s.b * P.deep + s.lvl; break;
    case PH_REC_W:
    case PH_REC_A: g = P.gL0 + s.sub; break;
    case PH_OBS_E: g = P.gHE; break;
    case PH_OBS_R: g = P.gR0 + s.sub; break;
    case PH_RK: g = s.rk_part; break;  // group 0 H_eff, group 1 H_drv
    default: return -1;
    }
    return P.e_g0[s.ens] + g;
}

// Slot holding the input vector of a trajectory's next matvec: psi, the normalised copy for
// the observables, or the RK stage argument.
__device__ __forceinline__ int src_slot(int phase, int cur, int rk_stage)
{
    if (phase == PH_RK) return rk_stage == 1 ? cur : kSlotArgs;
    return (phase == PH_OBS_E || phase == PH_OBS_R) ? (cur ^ 1) : cur;
}

// ---------------------------------------------------------------- RK propagator helpers
// E(t) of rk_right_part_dimer (core.cpp:11073-11103)
__device__ __forceinline__ double rk_drive(const Params &P, double t)
{
    if (P.drv_type == 1)
        return __dadd_rn(P.E0, __dmul_rn(P.A, sin(__dadd_rn(__dmul_rn(P.drv_freq, t), P.drv_phase))));
    const double mod_time = fmod(t, P.T), half_T = __dmul_rn(P.T, 0.5);
    return (mod_time < half_T) ? __dadd_rn(P.E0, P.A) : __dsub_rn(P.E0, P.A);
}

// Start time of step rk_sid of the current period (rk_period, core.cpp:446)
__device__ __forceinline__ double rk_step_time(const Params &P, const TrajState &s)
{
    return __dadd_rn(__dmul_rn((double)(P.period0 + s.pc), P.T), __dmul_rn((double)s.rk_sid, P.rk_step));
}

// Begin an RK step of size h from psi (slot cur) with norm prev; returns its first matvec's group.
__device__ __forceinline__ int rk_begin(TrajState &s, double h, double prev, int ctx)
{
    s.phase = PH_RK;
    s.rk_h = h;
    s.rk_prev = prev;
    s.rk_stage = 1;
    s.rk_part = 0;
    s.rk_ctx = ctx;
    return 0;
}

__device__ __forceinline__ void enqueue(const Params &P, int *cnt, int *list, int g, int tr)
{
    const int pos = atomicAdd(&cnt[g], 1);
    list[P.g_loff[g] + pos] = tr;
}

__device__ __forceinline__ void report_error(const Params &P, int tr, int code)
{
    if (atomicAdd(&P.ctrl[0], 1) == 0) {
        P.ctrl[1] = tr;
        P.ctrl[3] = code;
    }
}

// Counter bookkeeping after a completed step at level s.lvl (qj_proc.cpp:317-320, 330-338):
// advance the level's counter; a level that finished both steps returns to its parent,
// which undoes and redoes its own time advance (t -= dt; t += dt) and counts its step.
// Returns 0 inside a unit (two level-0 steps), 1 when a unit finished, 2 when the last unit
// of the last branch of a period finished.  A branch has brep units (1, or 2 deep_num_steps
// for the deep tasks, whose sub-period is two units: one_sub_period_deep, qj_proc.cpp:345-359).
__device__ __forceinline__ int advance(TrajState &s, const double *dt, int nb, int brep)
{
    int l = s.lvl;
    unsigned long long m = s.mask;
    while (true) {
        if (!((m >> l) & 1ull)) {
            m |= (1ull << l);
            s.lvl = l;
            s.mask = m;
            return 0;
        }
        m &= ~(1ull << l);
        if (l == 0) {
            s.mask = m;
            s.lvl = 0;
            if (++s.rk_sid < brep) return 1;
            s.rk_sid = 0;
            s.b += 1;
            if (s.b == nb) {
                s.b = 0;
                return 2;
            }
            return 1;
        }
        l -= 1;
        s.t = __dadd_rn(__dsub_rn(s.t, dt[l]), dt[l]);
    }
}

// |psi_k|^2 / norm as mult_scalar_double(mult_scalar_complex(phi, phi, 1), 1/norm).real
// (core.cpp:665-725), recomputed wherever it is needed (no scratch array)
__device__ __forceinline__ double adr_of(double2 v, double inv)
{
    return __dmul_rn(__dadd_rn(0.0, __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y))), inv);
}

// Observables of the state held in `col` (calc_chars_std[_start], core.cpp:665-725) and
// the normalised state psi / sqrt(norm) written to the spare slot for the energy and
// random-observable micro-steps.  Warp-cooperative; every lane computes the sequential
// sums identically.
__device__ void obs_prep(const Params &P, const TrajState &s, int tr, const double2 *col, int lane, int dump,
                         int is_start)
{
    const int d = dim_of(P, s);
    const double nrm = warp_norm(col, d, lane);
    const double sq = __dsqrt_rn(nrm);
    const double inv = __ddiv_rn(1.0, nrm);
    double2 *hat = slot_ptr(P, s.cur ^ 1, tr);
    double *adr_out = !P.o_adr ? nullptr
                      : (P.keep_adr ? P.o_adr + ((size_t)dump * P.n + tr) * P.d : P.o_adr + (size_t)tr * P.d);
    for (int k = lane; k < d; k += 32) {
        const double2 v = col[k];
        hat[k] = make_double2(__ddiv_rn(v.x, sq), __ddiv_rn(v.y, sq));
        if (adr_out) adr_out[k] = adr_of(v, inv);
    }
    double mean = 0.0;
    for (int k = lane; k < d; k += 32) mean = __dadd_rn(mean, __dmul_rn((double)k, adr_of(col[k], inv)));
    mean = warp_allsum(mean);
    const double ms = is_start ? mean : P.mean_start[tr];
    const double disp = __dmul_rn(__dsub_rn(mean, ms), __dsub_rn(mean, ms));
    double m2 = 0.0;
    for (int k = lane; k < d; k += 32) {
        const double dk = __dsub_rn((double)k, mean);
        m2 = __dadd_rn(m2, __dmul_rn(__dmul_rn(dk, dk), adr_of(col[k], inv)));
    }
    m2 = warp_allsum(m2);
    if (lane == 0) {
        const size_t o = (size_t)dump * P.n + tr;
        if (is_start) P.mean_start[tr] = mean;
        P.o_norm[o] = nrm;
        P.o_mean[o] = mean;
        P.o_disp[o] = disp;
        P.o_m2[o] = m2;
    }
    __syncwarp();
}

// Continue after a completed split step: period / dump / target bookkeeping.  Returns the
// next group, or -1 when the trajectory is done for this call.
__device__ int after_step(const Params &P, TrajState &s, int tr, const double2 *col, int lane)
{
    const int a = advance(s, dt_of(P, s), P.nb, P.brep);
    if (a == 2) s.pc += 1;
    if (a >= 1 && P.subdump && (s.rk_sid & 1) == 0) {  // deep task: a sub-period ended
        obs_prep(P, s, tr, col, lane, P.dump_base + s.di, 0);
        s.phase = PH_OBS_E;
        return P.gHE;
    }
    if (a == 2) {
        if (s.di < P.n_dumps && s.pc == P.dump_at[s.di]) {
            obs_prep(P, s, tr, col, lane, P.dump_base + s.di, 0);
            s.phase = PH_OBS_E;
            return P.gHE;
        }
        if (s.pc >= P.target) {
            s.phase = PH_DONE;
            return -1;
        }
    }
    return s.b * P.deep + s.lvl;
}

__device__ int finish_obs(const Params &P, TrajState &s)
{
    s.di += 1;
    if (s.pc >= P.target || (P.sub_target > 0 && s.di >= P.sub_target)) {
        s.phase = PH_DONE;
        return -1;
    }
    if (P.prop == 1) {  // next RK step of the period
        s.t = rk_step_time(P, s);
        return rk_begin(s, P.rk_step, s.rk_prev, 0);
    }
    s.phase = PH_STEP;
    return s.b * P.deep + s.lvl;
}

// An RK step finished without crossing (rk_period, core.cpp:443-449): next step, period and dump
// bookkeeping.  `col` holds psi, nrm its norm.
__device__ int rk_after_step(const Params &P, TrajState &s, int tr, const double2 *col, int lane,
                             double nrm)
{
    s.rk_prev = nrm;
    s.rk_sid += 1;
    if (s.rk_sid == P.rk_ns) {
        s.rk_sid = 0;
        s.pc += 1;
        if (s.di < P.n_dumps && s.pc == P.dump_at[s.di]) {
            obs_prep(P, s, tr, col, lane, P.dump_base + s.di, 0);
            s.phase = PH_OBS_E;
            return P.gHE;
        }
        if (s.pc >= P.target) {
            s.phase = PH_DONE;
            return -1;
        }
    }
    s.t = rk_step_time(P, s);
    return rk_begin(s, P.rk_step, nrm, 0);
}

// Apply the chosen jump channel: psi = (L_idx psi_hat) / sqrt(w_idx / g_idx)
// (experiment.cpp:1346-1369), record the channel, redraw eta (qj_proc.cpp:310-314) and
// count the finest-level step.
__device__ int apply_jump(const Params &P, TrajState &s, int tr, double2 *col, int lane, int idx,
                          double w_idx, int *err)
{
    const int d = dim_of(P, s);
    const double q = __dsqrt_rn(__ddiv_rn(w_idx, rate_of(P, s, idx)));
    double2 *dst = slot_ptr(P, s.cur ^ 1, tr);
    for (int k = lane; k < d; k += 32) {
        const double2 v = col[k];
        const double2 r = make_double2(__ddiv_rn(v.x, q), __ddiv_rn(v.y, q));
        dst[k] = r;
        col[k] = r;
    }
    __syncwarp();
    s.cur ^= 1;
    if (P.record && lane == 0) P.r_type[(size_t)(s.nrec - 1) * P.n + tr] = idx;
    s.eta = draw(P, tr, s, err);
    while (s.eta == 0.0 && *err == 0) s.eta = draw(P, tr, s, err);
    if (*err) return -1;
    if (P.prop == 1) {  // the end part of the interrupted RK step (rk_step_dimer, core.cpp:11946)
        const double nrm = warp_norm(col, d, lane);
        return rk_begin(s, s.rk_end, nrm, 0);
    }
    s.phase = PH_STEP;
    s.t = __dadd_rn(s.t, dt_of(P, s)[P.deep - 1]);
    return after_step(P, s, tr, col, lane);
}

// Warp-cooperative epilogue of one trajectory column: `col` holds M_g * psi in shared memory,
// `s_in` the trajectory's state record (loaded by the caller).  Returns the bucket of the
// trajectory's next micro-step, or -1 (done, paused or failed); the caller appends it.
__device__ int column_epilogue(const Params &P, double2 *col, int tr, const TrajState &s_in, int lane)
{
    const int d = dim_of(P, s_in);
    TrajState s = s_in;
    int g2 = -1;
    int err = 0;
    bool paused = false;

    switch (s.phase) {
    case PH_STEP: {
        const double nrm = warp_norm(col, d, lane);
        // is_norm_crossed throws (experiment.cpp:1247-1251); the split-precision form allows its
        // matvec rounding (a few 1e-6 of the norm) above 1 before calling it an error
        if (nrm > (P.split ? 1.0 + kSplitNormSlack : 1.0)) {
            err = ERR_NORM;
            break;
        }
        // split form: a norm within the split error of the threshold is not decided here; the
        // same step is computed again in FP64 and decides (the recheck itself clears the flag)
        const bool rechecked = s.rechk != 0;
        s.rechk = 0;
        if (P.split && P.recheck_tol > 0.0 && !rechecked && fabs(nrm - s.eta) <= P.recheck_tol * nrm) {
            s.rechk = 1;
            g2 = kRecheck;
            break;
        }
        const double dt = dt_of(P, s)[s.lvl];
        if (nrm > s.eta) {  // not crossed: accept psi' (qj_proc.cpp:317, 335)
            double2 *dst = slot_ptr(P, s.cur ^ 1, tr);
            for (int k = lane; k < d; k += 32) dst[k] = col[k];
            s.cur ^= 1;
            s.t = __dadd_rn(s.t, dt);
            g2 = after_step(P, s, tr, col, lane);
        } else if (s.lvl < P.deep - 1) {  // crossed on a coarse level: bisect from psi (qj_proc.cpp:328-331)
            s.lvl += 1;
            g2 = s.b * P.deep + s.lvl;
        } else {  // crossed on the finest level: jump (qj_proc.cpp:294-315)
            if (P.record) {
                if (s.nrec >= P.rec_cap) {  // record buffer full: hold here, host drains and resumes
                    paused = true;
                    break;
                }
                if (lane == 0) {
                    const size_t o = (size_t)s.nrec * P.n + tr;
                    P.r_time[o] = __dadd_rn(s.t, dt);
                    P.r_norm[o] = nrm;
                    P.r_eta[o] = s.eta;
                    P.r_type[o] = -1;
                }
                s.nrec += 1;
                s.jumps += 1;
            }
            // recovery: psi' /= sqrt(norm_square(psi'))  (experiment.cpp:1291-1296)
            const double sq = __dsqrt_rn(nrm);
            double2 *dst = slot_ptr(P, s.cur ^ 1, tr);
            for (int k = lane; k < d; k += 32) {
                const double2 v = col[k];
                dst[k] = make_double2(__ddiv_rn(v.x, sq), __ddiv_rn(v.y, sq));
            }
            s.cur ^= 1;
            s.ran = draw(P, tr, s, &err);
            if (err) break;
            s.tmpw = 0.0;
            s.phase = PH_REC_W;
            s.sub = 0;
            g2 = P.gL0;
        }
    } break;

    case PH_REC_W: {  // gnorms[i] = norm_square(L_i psi_hat) * g[i]  (experiment.cpp:1301-1322)
        double w = warp_norm(col, d, lane);
        w = __dmul_rn(w, rate_of(P, s, s.sub));
        if (lane == 0) P.gn[(size_t)tr * P.nd + s.sub] = w;
        s.tmpw = __dadd_rn(s.tmpw, w);
        if (s.sub + 1 < P.nd) {
            s.sub += 1;
            g2 = P.gL0 + s.sub;
            break;
        }
        __syncwarp();
        // channel choice (experiment.cpp:1324-1344)
        const double *gn = P.gn + (size_t)tr * P.nd;
        double ran = __dmul_rn(s.ran, s.tmpw);
        // the index never passes nd - 1 (the reference's loop reads past the end when
        // nd == 1 and ran > gnorms[0], which its own draws cannot produce)
        int index = 0;
        while (index < P.nd - 1 && __dsub_rn(ran, gn[index]) > 0.0) {
            ran = __dsub_rn(ran, gn[index]);
            index++;
        }
        if (s.tmpw == 0.0) {
            err = ERR_ZERO_W;
            break;
        }
        for (int it = 0; gn[index] == 0.0; it++) {
            if (it > 2 * P.nd) { err = ERR_ZERO_W; break; }
            index = (index == 0) ? index + 1 : index - 1;
            if (index >= P.nd) { err = ERR_ZERO_W; break; }
        }
        if (err) break;
        if (P.nd == 1) {
            g2 = apply_jump(P, s, tr, col, lane, index, w, &err);
        } else {
            s.phase = PH_REC_A;
            s.sub = index;
            g2 = P.gL0 + index;
        }
    } break;

    case PH_REC_A: {
        const double w = P.gn[(size_t)tr * P.nd + s.sub];
        g2 = apply_jump(P, s, tr, col, lane, s.sub, w, &err);
    } break;

    case PH_RK: {  // one right-hand side of rk_int_dimer (core.cpp:11592-11619), col = M arg
        if (s.rk_part == 0) {  // H_eff arg, kept for the drive part
            double2 *dst = slot_ptr(P, kSlotND, tr);
            for (int k = lane; k < d; k += 32) dst[k] = col[k];
            s.rk_part = 1;
            g2 = 1;
            break;
        }
        // k = -i (H_eff arg + E H_drv arg)  (core.cpp:11106-11112)
        const double E = rk_drive(P, s.t);
        const double2 *nd = slot_ptr(P, kSlotND, tr);
        const double2 *phi = slot_ptr(P, s.cur, tr);
        const double h = s.rk_h;
        if (s.rk_stage < 4) {
            // arg_upd (rk_proc.cpp:146-185) uses the full rk_step, also inside a begin or end part
            const double c = (s.rk_stage == 3) ? __dmul_rn(1.0, P.rk_step) : __dmul_rn(0.5, P.rk_step);
            double2 *kd = slot_ptr(P, kSlotK1 + s.rk_stage - 1, tr);
            double2 *args = slot_ptr(P, kSlotArgs, tr);
            for (int k = lane; k < d; k += 32) {
                const double2 a = nd[k], b = col[k], x = phi[k];
                const double kr = __dadd_rn(a.y, __dmul_rn(E, b.y)), ki = -__dadd_rn(a.x, __dmul_rn(E, b.x));
                kd[k] = make_double2(kr, ki);
                args[k] = make_double2(__dadd_rn(x.x, __dmul_rn(c, kr)), __dadd_rn(x.y, __dmul_rn(c, ki)));
            }
            if (s.rk_stage != 2) s.t = __dadd_rn(s.t, __dmul_rn(h, 0.5));
            s.rk_stage += 1;
            s.rk_part = 0;
            g2 = 0;
            break;
        }
        if (s.rk_ctx == 1 && P.record && s.nrec >= P.rec_cap) {  // record buffer full: hold here
            paused = true;
            break;
        }
        // rk_final (rk_proc.cpp:187-196): psi + (k1 + 2 k2 + 2 k3 + k4) h / 6, into col
        const double2 *k1 = slot_ptr(P, kSlotK1, tr), *k2 = slot_ptr(P, kSlotK1 + 1, tr);
        const double2 *k3 = slot_ptr(P, kSlotK1 + 2, tr);
        for (int k = lane; k < d; k += 32) {
            const double2 a = nd[k], b = col[k], x = phi[k], p1 = k1[k], p2 = k2[k], p3 = k3[k];
            const double kr = __dadd_rn(a.y, __dmul_rn(E, b.y)), ki = -__dadd_rn(a.x, __dmul_rn(E, b.x));
            const double sr = __dadd_rn(__dadd_rn(__dadd_rn(p1.x, __dmul_rn(2.0, p2.x)), __dmul_rn(2.0, p3.x)), kr);
            const double si = __dadd_rn(__dadd_rn(__dadd_rn(p1.y, __dmul_rn(2.0, p2.y)), __dmul_rn(2.0, p3.y)), ki);
            col[k] = make_double2(__dadd_rn(x.x, __ddiv_rn(__dmul_rn(sr, h), 6.0)),
                                  __dadd_rn(x.y, __ddiv_rn(__dmul_rn(si, h), 6.0)));
        }
        __syncwarp();
        const double nrm = warp_norm(col, d, lane);
        if (s.rk_ctx == 0) {
            if (nrm > 1.0) {  // is_norm_crossed throws (experiment.cpp:1247-1251)
                err = ERR_NORM;
                break;
            }
            if (nrm > s.eta) {  // not crossed: accept psi in place
                double2 *dst = slot_ptr(P, s.cur, tr);
                for (int k = lane; k < d; k += 32) dst[k] = col[k];
                g2 = rk_after_step(P, s, tr, col, lane, nrm);
            } else {  // crossed: integrate the begin part from psi, still in its slot (core.cpp:11913-11922)
                const double norm_diff = __dsub_rn(s.rk_prev, nrm);
                const double begin_part = __ddiv_rn(__dsub_rn(s.rk_prev, s.eta), norm_diff);
                const double end_part = __dsub_rn(1.0, begin_part);
                s.rk_end = __dmul_rn(h, end_part);
                s.t = __dsub_rn(s.t, h);
                g2 = rk_begin(s, __dmul_rn(h, begin_part), s.rk_prev, 1);
            }
        } else {  // begin part done: record the jump, rk_recovery (rk_proc.cpp:198-305)
            if (P.record) {
                if (lane == 0) {
                    const size_t o = (size_t)s.nrec * P.n + tr;
                    P.r_time[o] = s.t;
                    P.r_norm[o] = nrm;
                    P.r_eta[o] = s.eta;
                    P.r_type[o] = -1;
                }
                s.nrec += 1;
                s.jumps += 1;
            }
            const double sq = __dsqrt_rn(nrm);
            double2 *dst = slot_ptr(P, s.cur ^ 1, tr);
            for (int k = lane; k < d; k += 32) {
                const double2 v = col[k];
                dst[k] = make_double2(__ddiv_rn(v.x, sq), __ddiv_rn(v.y, sq));
            }
            s.cur ^= 1;
            s.ran = draw(P, tr, s, &err);
            if (err) break;
            s.tmpw = 0.0;
            s.phase = PH_REC_W;
            s.sub = 0;
            g2 = P.gL0;
        }
    } break;

    case PH_OBS_E: {  // energy <psi_hat| H + E0 Hd |psi_hat>  (experiment.cpp:1423-1469)
        const double2 *hat = slot_ptr(P, s.cur ^ 1, tr);
        double e = 0.0;
        for (int k = lane; k < d; k += 32) {
            const double2 h = hat[k], m = col[k];
            e = __dadd_rn(e, __dadd_rn(__dmul_rn(h.x, m.x), __dmul_rn(h.y, m.y)));
        }
        e = warp_allsum(e);
        if (lane == 0) P.o_energy[(size_t)(P.dump_base + s.di) * P.n + tr] = e;
        __syncwarp();
        if (P.nr > 0) {
            s.phase = PH_OBS_R;
            s.sub = 0;
            g2 = P.gR0;
        } else {
            g2 = finish_obs(P, s);
        }
    } break;

    case PH_OBS_R: {  // <psi_hat| R |psi_hat>  (experiment.cpp:2037-2068)
        const double2 *hat = slot_ptr(P, s.cur ^ 1, tr);
        double rr = 0.0, ri = 0.0;
        for (int k = lane; k < d; k += 32) {
            const double2 h = hat[k], m = col[k];
            const double cr = h.x, ci = -h.y;
            rr = __dadd_rn(rr, __dsub_rn(__dmul_rn(cr, m.x), __dmul_rn(ci, m.y)));
            ri = __dadd_rn(ri, __dadd_rn(__dmul_rn(ci, m.x), __dmul_rn(cr, m.y)));
        }
        rr = warp_allsum(rr);
        ri = warp_allsum(ri);
        if (lane == 0) P.o_robs[((size_t)(P.dump_base + s.di) * P.n + tr) * P.nr + s.sub] = make_double2(rr, ri);
        __syncwarp();
        if (s.sub + 1 < P.nr) {
            s.sub += 1;
            g2 = P.gR0 + s.sub;
        } else {
            g2 = finish_obs(P, s);
        }
    } break;

    default: break;
    }

    if (err || paused) g2 = -1;
    const bool to_recheck = (g2 == kRecheck);
    if (to_recheck) g2 = -1;
    if (lane == 0) {
        if (err) {
            s.err = err;
            s.phase = PH_ERROR;
            report_error(P, tr, err);
        } else if (paused) {
            s.paused = 1;
            atomicAdd(&P.ctrl[2], 1);
        }
        P.st[tr] = s;
    }
    __syncwarp();
    if (to_recheck) return kRecheck;
    return g2 >= 0 ? P.e_g0[s.ens] + g2 : -1;  // local group -> the ensemble's bucket
}

// Appends trajectories trs[c] to their next buckets g2s[c] (c < ncol, -1 skips) with one global
// atomic per distinct bucket of each 32 columns: warp w takes columns 32w .. 32w + 31, lanes
// with the same bucket find each other with __match_any_sync, the lowest reserves the run and
// the others take consecutive slots in lane order.  Independent of the number of groups.
__device__ void enqueue_batch(const Params &P, int *cnt_next, int *list_next, const int *trs, const int *g2s, int ncol)
{
    const int lane = threadIdx.x & 31;
    for (int c0 = (threadIdx.x >> 5) * 32; c0 < ncol; c0 += blockDim.x) {
        const int c = c0 + lane;
        const int g = (c < ncol) ? g2s[c] : -1;
        const unsigned m = __match_any_sync(0xffffffffu, g);
        const int leader = __ffs(m) - 1;
        int base = 0;
        if (g >= 0 && lane == leader) base = atomicAdd(&cnt_next[g], __popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (g >= 0) list_next[P.g_loff[g] + base + __popc(m & ((1u << lane) - 1u))] = trs[c];
    }
}

// Copies a 96-byte trajectory record with 16-byte accesses.
__device__ __forceinline__ void load_state(TrajState *dst, const TrajState *src)
{
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
    uint4 *t = reinterpret_cast<uint4 *>(dst);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(TrajState) / 16); i++) t[i] = s[i];
}

// Accumulates M_g * B for one sub-tile of NTE x TX columns (all rows), streaming the
// propagator in K-slabs through the TMA pipeline, then stages the result in Bt.
// Per output the k-ascending fma chain of the oracle is kept; within one k the four fmas
// are issued in two passes (re += Mr xr, im += Mr xi for every output, then re -= Mi xi,
// im += Mi xr), which leaves each chain's order unchanged.
__device__ __forceinline__ double neg(double x)
{
    return __longlong_as_double(__double_as_longlong(x) ^ (long long)0x8000000000000000ull);
}

// FP64 tensor-core MMA D = A(8x4) B(4x8) + D.  On sm_100a its accumulation equals the
// sequential chain fma(a3,b3, fma(a2,b2, fma(a1,b1, fma(a0,b0,c)))) bit for bit (checked on
// the device against that chain, the reverse chain and a single rounding), which is the
// oracle's per-output k-ascending order.
__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// Complex sub-tile product on the FP64 tensor core.  Rows are in 8-row blocks (RB of them,
// MD = 8 RB), columns in 8-column blocks (CB active of 4).  For one pair of complex k the
// real parts use A = [Mr_k, -Mi_k, Mr_k+1, -Mi_k+1] against B = [xr_k; xi_k; xr_k+1; xi_k+1]
// and the imaginary parts A = [Mr_k, Mi_k, ...] against B = [xi_k; xr_k; ...]; that is the
// k-ascending chain re += Mr xr; re -= Mi xi; im += Mr xi; im += Mi xr of the contract.
// WPC warps share one column block; warp `sub` of them owns row blocks sub, sub + WPC, ...
template <int NRB, int WPC>
__device__ __forceinline__ bool tile_dmma(const double2 *mat, double2 *Bt, double2 *Us, uint64_t *bar,
                                          int *released, uint32_t &phase, int d, int kp, int KB, int RB, int MD,
                                          int S16, int warp, int lane, int tid)
{
    const int g = lane >> 2, t = lane & 3;
    // warp w runs on scheduler w % 4; rotating the row-block index by column block gives
    // each scheduler the same number of row blocks
    const int cb = warp / WPC, sub = (warp % WPC + cb * (WPC / 4)) % WPC;
    const int th = t >> 1, todd = t & 1;
    const int nslab = (kp + KB - 1) / KB;
    bool ok = true;
    double re[NRB][2], im[NRB][2];
#pragma unroll
    for (int i = 0; i < NRB; i++) re[i][0] = re[i][1] = im[i][0] = im[i][1] = 0.0;

    if (!mbar_wait_bounded(&bar[kStages], (phase >> kStages) & 1u, kWaitLimit)) ok = false;
    phase ^= 1u << kStages;
    const double2 *bcol = Bt + (8 * cb + g) * S16;
    for (int sl = 0; sl < nslab; sl++) {
        const int q = sl % kStages;
        if (!mbar_wait_bounded(&bar[q], (phase >> q) & 1u, kWaitLimit)) ok = false;
        phase ^= 1u << q;
        const int k0 = sl * KB;
        const int kc = min(KB, kp - k0);  // even
        const double *Uq = reinterpret_cast<const double *>(Us + q * KB * MD);
#pragma unroll 2
        for (int kk = 0; kk < kc; kk += 2) {
            const double2 xb = bcol[k0 + kk + th];
            const double bre = todd ? xb.y : xb.x;
            const double bim = todd ? xb.x : xb.y;
            const double *urow = Uq + 2 * (size_t)(kk + th) * MD + todd;
#pragma unroll
            for (int i = 0; i < NRB; i++) {
                const int rb = sub + WPC * i;
                if (rb < RB) {
                    const double v = urow[2 * (8 * rb + g)];
                    dmma(re[i][0], re[i][1], todd ? neg(v) : v, bre);
                    dmma(im[i][0], im[i][1], v, bim);
                }
            }
        }
        // release the stage: the last of the 16 warps to finish it issues the refill, so no
        // warp waits for another's release (no CTA-wide barrier per slab)
        __syncwarp();
        if (lane == 0 && sl + kStages < nslab) {
            __threadfence_block();
            if (atomicAdd(&released[q], 1) == kThreads / 32 - 1) {
                released[q] = 0;
                const int sn = sl + kStages;
                const int kn = min(KB, kp - sn * KB);
                fence_proxy_async();
                mbar_expect_tx(&bar[q], (uint32_t)(kn * MD * 16));
                bulk_g2s(Us + q * KB * MD, mat + (size_t)sn * KB * MD, (uint32_t)(kn * MD * 16), &bar[q]);
            }
        }
        __syncwarp();  // lanes 1-31 wait here, not spinning on the next slab beside the issuing lane
    }
    __syncthreads();
    // stage: thread (g, t) of row block rb holds rows 8 rb + g, columns 8 cb + 2t, 8 cb + 2t + 1
#pragma unroll
    for (int i = 0; i < NRB; i++) {
        const int rb = sub + WPC * i;
        const int row = 8 * rb + g;
        if (rb < RB && row < d) {
            Bt[(8 * cb + 2 * t) * S16 + row] = make_double2(re[i][0], im[i][0]);
            Bt[(8 * cb + 2 * t + 1) * S16 + row] = make_double2(re[i][1], im[i][1]);
        }
    }
    return ok;
}

// Estimated cost of a bucket of m columns cut into sub-tiles the way the kernel cuts them
// (32-column chunks; a rest of 17..24 columns as 16 + rest), in units of ~5k cycles: 2 per
// sub-tile (gather, epilogue), 6 per active 8-column block (MMA loop), and 3 more per
// sub-tile of the jump-operator and observable buckets, whose epilogues renormalise, draw
// and reduce.
// Columns of the next sub-tile of a bucket piece of m columns: with 32-column sub-tiles a rest
// of 17..24 columns is cut as 16 + rest (no sub-tile of 3 column blocks); narrower sub-tiles
// (large d) take min(m, NC).
__device__ __forceinline__ int subtile_cols(int m, int NC)
{
    if (NC == kNC) return (m > 24) ? min(m, kNC) : (m > 16 ? 16 : m);
    return min(m, NC);
}

__device__ __forceinline__ int subtile_cost(int m, int NC, int u_sub, int u_blk, int u_col4)
{
    int c = 0;
    while (m > 0) {
        const int s = subtile_cols(m, NC);
        const int cb = (s + 7) / 8;
        c += u_sub + u_blk * ((cb == 3) ? 4 : cb) + (s * u_col4) / 4;
        m -= s;
    }
    return c;
}

// Estimated cost of group g's bucket of m columns, in units of 0.25 us at d = 201, fitted to the
// busy time of every CTA in 512 full micro-steps of the headline ensemble against the work it
// got (least squares, 1.9 us rms): 7.8 us per sub-tile (gather, slab pipeline fill, epilogue
// passes), 15.0 us per active 8-column block (MMA loop), 0.06 us per column and 0.15 us more per
// column of the jump-operator and observable buckets (their epilogues renormalise, draw and
// reduce); scaled to the group's dimension (epilogue ~ d, MMA ~ row blocks x k rows).
__device__ __forceinline__ int group_cost(const Params &P, int g, int m)
{
    if (m == 0) return 0;
    const int e = P.g_ens[g], d = P.e_d[e];
    const bool heavy = g - P.e_g0[e] >= P.gL0;
    const int u_sub = max(1, (31 * d + 100) / 201);
    const int u_blk = max(1, (((d + 7) >> 3) * ((d + 1) & ~1) * 60 + 2626) / 5252);
    const int u_col4 = max(1, ((heavy ? 7 : 2) * d + 200) / 402);
    return subtile_cost(m, P.e_nc[e], u_sub, u_blk, u_col4);
}

// Plan of a micro-step from its bucket sizes cnt[G]: bucket starts plan[0..G] and cost prefix
// plan[G+1..2G+1].  Block-wide (any multiple of 32 threads); reads cnt past L1 (its atomics
// were made by other CTAs).
__device__ void plan_scan(const Params &P, const int *cnt)
{
    __shared__ int w_c[32], w_k[32];
    const int G = P.G, nt = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int per = (G + nt - 1) / nt;
    const int g0 = min(G, tid * per), g1 = min(G, g0 + per);
    int c = 0, k = 0;
    for (int g = g0; g < g1; g++) {
        const int m = __ldcg(cnt + g);
        c += m;
        k += group_cost(P, g, m);
    }
    int ic = c, ik = k;  // inclusive warp scans
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int yc = __shfl_up_sync(0xffffffffu, ic, off), yk = __shfl_up_sync(0xffffffffu, ik, off);
        if (lane >= off) {
            ic += yc;
            ik += yk;
        }
    }
    if (lane == 31) {
        w_c[warp] = ic;
        w_k[warp] = ik;
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = nt >> 5;
        int vc = lane < nw ? w_c[lane] : 0, vk = lane < nw ? w_k[lane] : 0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int yc = __shfl_up_sync(0xffffffffu, vc, off), yk = __shfl_up_sync(0xffffffffu, vk, off);
            if (lane >= off) {
                vc += yc;
                vk += yk;
            }
        }
        if (lane < nw) {
            w_c[lane] = vc;  // inclusive totals through warp `lane`
            w_k[lane] = vk;
        }
    }
    __syncthreads();
    int cs = ic - c + (warp ? w_c[warp - 1] : 0), ks = ik - k + (warp ? w_k[warp - 1] : 0);
    for (int g = g0; g < g1; g++) {
        const int m = __ldcg(cnt + g);
        P.plan[g] = cs;
        P.plan[G + 1 + g] = ks;
        cs += m;
        ks += group_cost(P, g, m);
    }
    if (tid == nt - 1) {
        P.plan[G] = cs;
        P.plan[2 * G + 1] = ks;
    }
    __syncthreads();
}

// Column position of cost offset k (monotone in k) in a plan.
__device__ __forceinline__ int cost_to_column(const int *cstart, const int *kc, int G, long long k)
{
    if (k >= kc[G]) return cstart[G];
    int lo = 0, hi = G;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (kc[mid] <= k) lo = mid;
        else hi = mid;
    }
    const int cnt = cstart[lo + 1] - cstart[lo];
    const int cost = kc[lo + 1] - kc[lo];
    if (cost <= 0) return cstart[lo];
    const long long off = (k - kc[lo]) * (long long)cnt / cost;
    const int col = (int)min((long long)cnt, ((off + 4) / 8) * 8);
    return cstart[lo] + col;
}

// One lock-step micro-step: grouped complex GEMM over the buckets of step `s` on the FP64
// tensor core, with the fused epilogue.  The concatenated bucket lists (C columns) are split
// into equal column ranges, one per persistent CTA; each range is processed as sub-tiles of
// at most 32 columns of one matrix, and a sub-tile costs in proportion to its active 8-column
// blocks (1, 2 or 4): the warps are spread over the row blocks of the active column blocks.
// Each ensemble has its own sub-tile width (32, 16 or 8 columns) and slab height; the shared
// memory holds the staged columns (stride MD + 1, odd: conflict-free column reads) followed by
// the propagator slabs, laid out per sub-tile.  R4, R2, R1: row blocks per warp of the sub-tiles
// with 4, 2 and 1 column blocks (4, 8 and 16 warps per column block), large enough for every
// ensemble that uses them.
template <int R4, int R2, int R1>
__global__ void __launch_bounds__(kThreads, 1) step_kernel(const Params P, int s)
{
    extern __shared__ __align__(128) unsigned char smem[];
    double2 *Bt = reinterpret_cast<double2 *>(smem);
    __shared__ __align__(8) uint64_t bar[kStages + 1];
    __shared__ int released[kStages];
    __shared__ int s_tr[kNC];
    __shared__ long long s_src[kNC];
    __shared__ __align__(16) TrajState s_st[kNC];
    __shared__ int s_g2[kNC];
    __shared__ int s_last;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int G = P.G, n = P.n;
    int *cnt_next = P.cnt + ((s + 1) % 3) * G;
    const int *list_cur = P.lists + (size_t)(s & 1) * P.ltot;
    int *list_next = P.lists + (size_t)((s + 1) & 1) * P.ltot;
    const int *cstart = P.plan, *kc = P.plan + G + 1;  // this step's plan

    if (blockIdx.x == 0)
        for (int i = tid; i < G; i += kThreads) P.cnt[((s + 2) % 3) * G + i] = 0;
    if (tid == 0) {
        for (int q = 0; q <= kStages; q++) mbar_init(&bar[q], 1);
        for (int q = 0; q < kStages; q++) released[q] = 0;
    }
    __syncthreads();
    // equal shares of the estimated cost, mapped back to column positions (8-column aligned
    // inside each bucket): buckets that split into many narrow sub-tiles get shorter ranges
    const long long K = kc[G];
    const int c_lo = cost_to_column(cstart, kc, G, K * blockIdx.x / gridDim.x);
    const int c_hi = cost_to_column(cstart, kc, G, K * (blockIdx.x + 1) / gridDim.x);
    uint32_t phase = 0;
    long long work = 0;
    long long tr_setup = 0, tr_loop = 0, tr_epi = 0, tr_sub = 0, tr_cb = 0;
    const long long t_begin = clock64();

    for (int pos = c_lo; pos < c_hi;) {
        const long long t0 = clock64();
        int lo = 0, hi = G;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (cstart[mid] <= pos) lo = mid;
            else hi = mid;
        }
        const int g = lo;
        const int idx = pos - cstart[g];
        // the group's matrix: its ensemble's dimension, padded rows, k rows and tiling
        const int eg = P.g_ens[g];
        const int dg = P.e_d[eg];
        const int MD = 8 * ((dg + 7) / 8), RB = MD / 8, kp = (dg + 1) & ~1;
        const int S16 = MD + 1, KB = P.e_kb[eg], NC = P.e_nc[eg];
        double2 *Us = Bt + NC * S16;
        const int nslab = (kp + KB - 1) / KB;
        // piece of this group left in the range, cut so that no sub-tile has 3 column blocks
        const int m = min(c_hi - pos, cstart[g + 1] - pos);
        const int ncol = subtile_cols(m, NC);
        const int ncb = (ncol + 7) / 8;
        if (tid < kNC) {
            if (tid < ncol) {
                const int tr = list_cur[P.g_loff[g] + idx + tid];
                load_state(&s_st[tid], &P.st[tr]);
                const int slot = src_slot(s_st[tid].phase, s_st[tid].cur, s_st[tid].rk_stage);
                s_tr[tid] = tr;
                s_src[tid] = ((long long)slot * n + tr) * P.MD;
            } else {
                s_tr[tid] = -1;
            }
        }
        __syncthreads();
        const double2 *mat = P.mats + P.g_off[g];
        if (tid == 0) {
            fence_proxy_async();
            mbar_expect_tx(&bar[kStages], (uint32_t)(ncol * kp * 16));
            for (int c = 0; c < ncol; c++) bulk_g2s(Bt + c * S16, P.psi + s_src[c], (uint32_t)(kp * 16), &bar[kStages]);
            for (int q = 0; q < kStages && q < nslab; q++) {
                const int kcq = min(KB, kp - q * KB);
                mbar_expect_tx(&bar[q], (uint32_t)(kcq * MD * 16));
                bulk_g2s(Us + q * KB * MD, mat + (size_t)q * KB * MD, (uint32_t)(kcq * MD * 16), &bar[q]);
            }
        }
        __syncwarp();  // warp 0's other lanes wait for the copies to be issued instead of spinning on them
        const long long t1 = clock64();
        bool ok;
        if (ncb == 1)
            ok = tile_dmma<R1, 16>(mat, Bt, Us, bar, released, phase, dg, kp, KB, RB, MD, S16, warp, lane, tid);
        else if (ncb == 2)
            ok = tile_dmma<R2, 8>(mat, Bt, Us, bar, released, phase, dg, kp, KB, RB, MD, S16, warp, lane, tid);
        else
            ok = tile_dmma<R4, 4>(mat, Bt, Us, bar, released, phase, dg, kp, KB, RB, MD, S16, warp, lane, tid);
        if (!__syncthreads_and(ok ? 1 : 0)) {  // a bounded wait gave up: report and stop
            if (tid == 0) {
                atomicAdd(&P.ctrl[4], 1);
                report_error(P, -1, ERR_TIMEOUT);
            }
            break;
        }
        const long long t2 = clock64();
        for (int c = warp; c < ncol; c += kThreads / 32) {
            const int g2 = column_epilogue(P, Bt + c * S16, s_tr[c], s_st[c], lane);
            if (lane == 0) s_g2[c] = g2;
        }
        __syncthreads();
        enqueue_batch(P, cnt_next, list_next, s_tr, s_g2, ncol);
        work += ncol;
        pos += ncol;
        fence_proxy_async();
        __syncthreads();
        const long long t3 = clock64();
        tr_setup += t1 - t0;
        tr_loop += t2 - t1;
        tr_epi += t3 - t2;
        tr_sub += 1;
        tr_cb += (ncb == 3) ? 4 : ncb;
    }
    if (tid == 0 && work) atomicAdd((unsigned long long *)P.work, (unsigned long long)work);
    if (P.trace && tid == 0) {
        long long *t = P.trace + (size_t)blockIdx.x * kTraceFields;
        t[0] += clock64() - t_begin;
        t[1] += tr_setup;
        t[2] += 0;
        t[3] += tr_loop;
        t[4] += tr_epi;
        t[5] += tr_sub;
        t[6] += tr_cb;
        t[7] += work;
    }
    // the last CTA to finish plans the next micro-step from the buckets all CTAs filled
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        s_last = atomicAdd(P.plan_sync, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        plan_scan(P, cnt_next);
        if (tid == 0) *P.plan_sync = 0u;
    }
}

// Plan of step 0 after a host-side enqueue (schedule, observe, resume): one block.
__global__ void __launch_bounds__(1024) plan_kernel(const Params P)
{
    plan_scan(P, P.cnt);
}

// Bucket trajectories for step 0 of a call.  mode 0: start of a run of P.target periods;
// mode 1: resume trajectories paused on a full record buffer; mode 2: continue a deep task from
// where the previous call stopped (a sub-period boundary: branch, unit and period count kept).
__global__ void schedule_kernel(const Params P, int mode)
{
    const int tr = blockIdx.x * blockDim.x + threadIdx.x;
    if (tr >= P.n) return;
    TrajState s = P.st[tr];
    if (s.phase == PH_ERROR) return;
    if (mode == 0) {
        s.pc = 0;
        s.di = 0;
        s.b = 0;
        s.lvl = 0;
        s.mask = 0;
        s.rk_sid = 0;
        s.paused = 0;
        s.phase = (P.target > 0 && runs(P, tr)) ? PH_STEP : PH_DONE;
    } else if (mode == 2) {
        s.di = 0;
        s.paused = 0;
        s.phase = (P.sub_target > 0 && runs(P, tr)) ? PH_STEP : PH_DONE;
    } else {
        if (!s.paused) return;
        s.paused = 0;
    }
    const int g = group_of(P, s);
    if (g >= 0) enqueue(P, P.cnt, P.lists, g, tr);
    P.st[tr] = s;
}

// Host-initiated observables of the current states (one warp per trajectory); the energy
// and random-observable matvecs follow as micro-steps.
__global__ void observe_kernel(const Params P, int dump, int is_start)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tr = blockIdx.x * (blockDim.x / 32) + warp;
    if (tr >= P.n || (P.active && !P.active[tr])) return;
    double2 *col = reinterpret_cast<double2 *>(smem) + (size_t)warp * P.MD;
    TrajState s = P.st[tr];
    if (s.phase == PH_ERROR) return;
    const double2 *src = slot_ptr(P, s.cur, tr);
    for (int k = lane; k < dim_of(P, s); k += 32) col[k] = src[k];
    __syncwarp();
    obs_prep(P, s, tr, col, lane, dump, is_start);
    if (lane == 0) {
        s.pc = 0;
        s.di = 0;
        s.phase = PH_OBS_E;
        enqueue(P, P.cnt, P.lists, P.e_g0[s.ens] + P.gHE, tr);
        P.st[tr] = s;
    }
}

// ---------------------------------------------------------------- ensemble purity
// rho = (1/n) sum_tr psi_hat psi_hat^dagger over the current states, purity = ||rho||_F^2 (the
// formula of calc_purity, source/cpp/CQdiss/CQdiss/CalcTraseRO2.cpp:57-75, applied to the
// trajectory ensemble).  Canonical order, shared bit-for-bit with the CPU oracle: psi_hat =
// psi / sqrt(p) with the canonical 32-lane norm p; rho_ij accumulates trajectories in ascending
// order with fma (re += a_r b_r, re += a_i b_i, im += a_i b_r, im += -a_r b_i) and is divided by n;
// the purity is the canonical 32-lane squared norm of rho flattened row-major.
__global__ void normalize_kernel(const Params P, double2 *hat)
{
    const int lane = threadIdx.x & 31;
    const int tr = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (tr >= P.n) return;
    const double2 *src = slot_ptr(P, P.st[tr].cur, tr);
    const double q = __dsqrt_rn(warp_norm(src, P.d, lane));
    double2 *dst = hat + (size_t)tr * P.MD;
    for (int k = lane; k < P.d; k += 32) {
        const double2 v = src[k];
        dst[k] = make_double2(__ddiv_rn(v.x, q), __ddiv_rn(v.y, q));
    }
}

// one 16 x 16 tile of rho per block (256 threads), trajectories staged 32 at a time
__global__ void __launch_bounds__(256) rho_kernel(const Params P, const double2 *hat, double2 *rho)
{
    __shared__ double2 a[32][16], b[32][16];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int i0 = blockIdx.y * 16, j0 = blockIdx.x * 16;
    double re = 0.0, im = 0.0;
    for (int c = 0; c < P.n; c += 32) {
        for (int e = threadIdx.x; e < 32 * 16; e += 256) {
            const int t = e >> 4, k = e & 15, tr = c + t;
            double2 za = make_double2(0.0, 0.0), zb = za;
            if (tr < P.n) {
                if (i0 + k < P.d) za = hat[(size_t)tr * P.MD + i0 + k];
                if (j0 + k < P.d) zb = hat[(size_t)tr * P.MD + j0 + k];
            }
            a[t][k] = za;
            b[t][k] = zb;
        }
        __syncthreads();
        const int m = min(32, P.n - c);
        for (int t = 0; t < m; t++) {
            const double2 x = a[t][ty], y = b[t][tx];
            re = __fma_rn(x.x, y.x, re);
            re = __fma_rn(x.y, y.y, re);
            im = __fma_rn(x.y, y.x, im);
            im = __fma_rn(-x.x, y.y, im);
        }
        __syncthreads();
    }
    const int i = i0 + ty, j = j0 + tx;
    if (i < P.d && j < P.d)
        rho[(size_t)i * P.d + j] = make_double2(__ddiv_rn(re, (double)P.n), __ddiv_rn(im, (double)P.n));
}

__global__ void purity_kernel(const double2 *rho, int dd, double *out)
{
    const double s = warp_norm(rho, dd, threadIdx.x & 31);
    if (threadIdx.x == 0) *out = s;
}

__global__ void init_state_kernel(const Params P, int tr0, int tr1)
{
    const int tr = tr0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (tr >= tr1) return;
    TrajState s;
    s.t = 0.0;
    s.eta = 0.0;
    s.ran = 0.0;
    s.tmpw = 0.0;
    s.rng_pos = 0;
    s.mask = 0;
    s.lvl = 0;
    s.b = 0;
    s.phase = PH_DONE;
    s.cur = 0;
    s.sub = 0;
    s.pc = 0;
    s.di = 0;
    s.jumps = 0;
    s.nrec = 0;
    s.err = 0;
    s.paused = 0;
    s.rng_src = tr;
    s.rk_h = 0.0;
    s.rk_prev = 0.0;
    s.rk_end = 0.0;
    s.rk_sid = 0;
    s.rk_stage = 0;
    s.rk_part = 0;
    s.rk_ctx = 0;
    int lo = 0, hi = P.E;  // ensemble e with e_tr0[e] <= tr < e_tr0[e + 1]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (P.e_tr0[mid] <= tr) lo = mid;
        else hi = mid;
    }
    s.ens = lo;
    s.rechk = 0;
    // rows past the ensemble's dimension stay zero (they meet the zero rows of its matrices)
    double2 *psi0 = P.psi + (size_t)tr * P.MD;
    for (int k = P.e_d[lo]; k < P.MD; k++) psi0[k] = make_double2(0.0, 0.0);
    P.st[tr] = s;
}

// eta_0 draw of trans_process_single (experiment.cpp:3260-3265)
__global__ void thresholds_kernel(const Params P, int tr0, int tr1)
{
    const int tr = tr0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (tr >= tr1) return;
    TrajState s = P.st[tr];
    int err = 0;
    s.eta = 0.0;
    while (s.eta == 0.0 && err == 0) s.eta = draw(P, tr, s, &err);
    if (err) {
        s.err = err;
        s.phase = PH_ERROR;
        report_error(P, tr, err);
    }
    P.st[tr] = s;
}

__global__ void reset_times_kernel(const Params P)
{
    const int tr = blockIdx.x * blockDim.x + threadIdx.x;
    if (tr < P.n) P.st[tr].t = 0.0;
}

__global__ void clear_records_kernel(const Params P)
{
    const int tr = blockIdx.x * blockDim.x + threadIdx.x;
    if (tr < P.n) P.st[tr].nrec = 0;
}

// ---------------------------------------------------------------- host-side launchers
size_t step_smem_bytes(int MD, int nc, int kb);

template <int R4, int R2, int R1>
static cudaError_t launch_step_t(const Params &P, int s, int grid, cudaStream_t st)
{
    static int attr_bytes = 0;
    if (attr_bytes < P.step_smem) {
        cudaError_t e =
            cudaFuncSetAttribute(step_kernel<R4, R2, R1>, cudaFuncAttributeMaxDynamicSharedMemorySize, P.step_smem);
        if (e != cudaSuccess) return e;
        attr_bytes = P.step_smem;
    }
    step_kernel<R4, R2, R1><<<grid, kThreads, P.step_smem, st>>>(P, s);
    return cudaGetLastError();
}

cudaError_t launch_split_step(const Params &P, int s, int grid, cudaStream_t st);

// Instantiation for the largest padded rows MD: up to 256 rows every sub-tile width may occur
// (R4 = ceil(RB / 4)); up to 512 the 32-column sub-tiles belong to ensembles of at most 256 rows
// (R4 = 8) and R2 = ceil(RB / 8); up to 1024 also R2 = 8 and R1 = ceil(RB / 16).
cudaError_t launch_step(const Params &P, int s, int grid, cudaStream_t st)
{
    if (P.split) return launch_split_step(P, s, grid, st);
    const int RB = P.MD / 8;
    if (RB <= 32) {
        switch ((RB + 3) / 4) {
        case 1: return launch_step_t<1, 1, 1>(P, s, grid, st);
        case 2: return launch_step_t<2, 1, 1>(P, s, grid, st);
        case 3: return launch_step_t<3, 2, 1>(P, s, grid, st);
        case 4: return launch_step_t<4, 2, 1>(P, s, grid, st);
        case 5: return launch_step_t<5, 3, 2>(P, s, grid, st);
        case 6: return launch_step_t<6, 3, 2>(P, s, grid, st);
        case 7: return launch_step_t<7, 4, 2>(P, s, grid, st);
        default: return launch_step_t<8, 4, 2>(P, s, grid, st);
        }
    }
    if (RB <= 64) {
        switch ((RB + 7) / 8) {
        case 5: return launch_step_t<8, 5, 3>(P, s, grid, st);
        case 6: return launch_step_t<8, 6, 3>(P, s, grid, st);
        case 7: return launch_step_t<8, 7, 4>(P, s, grid, st);
        default: return launch_step_t<8, 8, 4>(P, s, grid, st);
        }
    }
    switch ((RB + 15) / 16) {
    case 5: return launch_step_t<8, 8, 5>(P, s, grid, st);
    case 6: return launch_step_t<8, 8, 6>(P, s, grid, st);
    case 7: return launch_step_t<8, 8, 7>(P, s, grid, st);
    case 8: return launch_step_t<8, 8, 8>(P, s, grid, st);
    default: return cudaErrorInvalidValue;
    }
}

// Padded rows for dimension d: whole 8-row blocks (the m8n8k4 row block).
int pick_layout(int d, int *rows_per_block)
{
    *rows_per_block = 8;
    return 8 * ((d + 7) / 8);
}

// Shared memory of the step kernel: nc staged columns of MD + 1 (odd stride) and kStages
// propagator slabs of kb k rows.
size_t step_smem_bytes(int MD, int nc, int kb)
{
    return (size_t)(nc * (MD + 1) + kStages * kb * MD) * sizeof(double2);
}

// Static shared memory of the step kernel (the same for every instantiation).
size_t step_static_smem()
{
    cudaFuncAttributes a{};
    if (cudaFuncGetAttributes(&a, step_kernel<1, 1, 1>) != cudaSuccess) return 16384;
    return a.sharedSizeBytes;
}

// Widest sub-tile (32, 16 or 8 columns) whose staged columns leave room for slabs of at least
// 8 k rows (at most 16, even) in `budget` bytes of dynamic shared memory, with at most 8 row
// blocks per warp; failing that, the widest with 2-row slabs.  Returns false when none fits.
bool pick_step_tiles(int MD, size_t budget, int *nc, int *kb)
{
    const int RB = MD / 8;
    for (int min_kb = 8; min_kb >= 2; min_kb -= 6) {
        for (int c = kNC; c >= 8; c /= 2) {
            const int W1 = 16 / (c / 8);
            if ((RB + W1 - 1) / W1 > 8) continue;
            const size_t bt = (size_t)c * (MD + 1) * sizeof(double2);
            if (bt >= budget) continue;
            int k = (int)((budget - bt) / ((size_t)kStages * MD * sizeof(double2)));
            k = std::min(k, kKB) & ~1;
            if (k < min_kb) continue;
            *nc = c;
            *kb = k;
            return true;
        }
    }
    return false;
}

// The first micro-step after a host-side enqueue needs its plan (both forms).
cudaError_t launch_split_plan(const Params &P, cudaStream_t st);

static cudaError_t launch_plan(const Params &P, cudaStream_t st)
{
    if (P.split) return launch_split_plan(P, st);
    plan_kernel<<<1, 1024, 0, st>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_schedule(const Params &P, int mode, cudaStream_t st)
{
    schedule_kernel<<<(P.n + 255) / 256, 256, 0, st>>>(P, mode);
    return launch_plan(P, st);
}

cudaError_t launch_observe(const Params &P, int dump, int is_start, cudaStream_t st)
{
    const size_t smem = (size_t)8 * P.MD * sizeof(double2);
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(observe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)(8 * kMaxMD * sizeof(double2)));
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    observe_kernel<<<(P.n + 7) / 8, 256, smem, st>>>(P, dump, is_start);
    return launch_plan(P, st);
}

cudaError_t launch_purity(const Params &P, double2 *hat, double2 *rho, double *out, cudaStream_t st)
{
    normalize_kernel<<<(P.n + 7) / 8, 256, 0, st>>>(P, hat);
    const int tiles = (P.d + 15) / 16;
    rho_kernel<<<dim3(tiles, tiles), 256, 0, st>>>(P, hat, rho);
    purity_kernel<<<1, 32, 0, st>>>(rho, P.d * P.d, out);
    return cudaGetLastError();
}

// Start of a run with the RK propagator: step 0 of the first period from psi (warp per trajectory).
__global__ void rk_schedule_kernel(const Params P)
{
    const int lane = threadIdx.x & 31;
    const int tr = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (tr >= P.n) return;
    TrajState s = P.st[tr];
    if (s.phase == PH_ERROR) return;
    const double nrm = warp_norm(slot_ptr(P, s.cur, tr), P.d, lane);
    s.pc = 0;
    s.di = 0;
    s.paused = 0;
    s.rk_sid = 0;
    if (P.target > 0 && runs(P, tr)) {
        s.t = rk_step_time(P, s);
        rk_begin(s, P.rk_step, nrm, 0);
        if (lane == 0) enqueue(P, P.cnt, P.lists, P.e_g0[s.ens], tr);
    } else {
        s.phase = PH_DONE;
    }
    if (lane == 0) P.st[tr] = s;
}

cudaError_t launch_rk_schedule(const Params &P, cudaStream_t st)
{
    rk_schedule_kernel<<<(P.n + 7) / 8, 256, 0, st>>>(P);
    return launch_plan(P, st);
}

cudaError_t launch_init_state(const Params &P, cudaStream_t st, int tr0, int tr1)
{
    if (tr1 < 0) tr1 = P.n;
    if (tr1 <= tr0) return cudaSuccess;
    init_state_kernel<<<(tr1 - tr0 + 255) / 256, 256, 0, st>>>(P, tr0, tr1);
    return cudaGetLastError();
}

cudaError_t launch_thresholds(const Params &P, cudaStream_t st, int tr0, int tr1)
{
    if (tr1 < 0) tr1 = P.n;
    if (tr1 <= tr0) return cudaSuccess;
    thresholds_kernel<<<(tr1 - tr0 + 255) / 256, 256, 0, st>>>(P, tr0, tr1);
    return cudaGetLastError();
}

cudaError_t launch_reset_times(const Params &P, cudaStream_t st)
{
    reset_times_kernel<<<(P.n + 255) / 256, 256, 0, st>>>(P);
    return cudaGetLastError();
}

// FP64 FMA throughput microbenchmark: 8 independent fma chains per thread.
__global__ void fp64_peak_kernel(double *out, int iters, double a, double b)
{
    double x[8];
#pragma unroll
    for (int i = 0; i < 8; i++) x[i] = threadIdx.x * 1e-9 + i;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = __fma_rn(x[i], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; i++) s += x[i];
    if (s == 12345.678) out[0] = s;  // keeps the chains live
}

// FP64 tensor-core throughput microbenchmark: 8 independent m8n8k4 accumulator chains per warp.
__global__ void dmma_peak_kernel(double *out, int iters, double a, double b)
{
    double c[8][2];
#pragma unroll
    for (int i = 0; i < 8; i++) c[i][0] = c[i][1] = threadIdx.x * 1e-9 + i;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++) dmma(c[i][0], c[i][1], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; i++) s += c[i][0] + c[i][1];
    if (s == 12345.678) out[0] = s;
}

cudaError_t launch_dmma_peak(double *out, int blocks, int iters, cudaStream_t st)
{
    dmma_peak_kernel<<<blocks, 256, 0, st>>>(out, iters, 1e-3, 1e-3);
    return cudaGetLastError();
}

cudaError_t launch_fp64_peak(double *out, int blocks, int iters, cudaStream_t st)
{
    fp64_peak_kernel<<<blocks, 256, 0, st>>>(out, iters, 0.9999999, 1e-7);
    return cudaGetLastError();
}

cudaError_t launch_clear_records(const Params &P, cudaStream_t st)
{
    clear_records_kernel<<<(P.n + 255) / 256, 256, 0, st>>>(P);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- split-precision form
#include "qjx_split.cuh"

cudaError_t launch_split_plan(const Params &P, cudaStream_t st)
{
    split_plan_kernel<<<1, 512, 0, st>>>(P, P.grid);
    return cudaGetLastError();
}

// Static shared memory of the split kernel.
size_t split_static_smem()
{
    cudaFuncAttributes a{};
    if (cudaFuncGetAttributes(&a, split_step_kernel) != cudaSuccess) return 32768;
    return a.sharedSizeBytes;
}

static cudaError_t split_smem_attr(size_t smem)
{
    static int attr_bytes = 0;
    if (attr_bytes < (int)smem) {
        cudaError_t e = cudaFuncSetAttribute(split_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_bytes = (int)smem;
    }
    return cudaSuccess;
}

cudaError_t launch_split_step(const Params &P, int s, int grid, cudaStream_t st)
{
    const size_t smem = split_smem_bytes(P.MDs, P.MD, P.sstages);
    cudaError_t e = split_smem_attr(smem);
    if (e != cudaSuccess) return e;
    split_step_kernel<<<grid, kThreads, smem, st>>>(P, s, 1);
    return cudaGetLastError();
}

// Micro-steps s0 .. s0 + nsteps - 1 in one launch (fewer when the work runs out first; the
// count is left in P.sdone): a cooperative launch, so that every CTA is resident for the grid
// barriers between the steps.
cudaError_t launch_split_steps(const Params &P, int s0, int nsteps, int grid, cudaStream_t st)
{
    const size_t smem = split_smem_bytes(P.MDs, P.MD, P.sstages);
    cudaError_t e = split_smem_attr(smem);
    if (e != cudaSuccess) return e;
    Params Pc = P;
    void *args[] = {&Pc, &s0, &nsteps};
    return cudaLaunchCooperativeKernel((const void *)split_step_kernel, dim3(grid), dim3(kThreads), args, smem, st);
}

}  // namespace qjx
