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
//     (cp.async.bulk + mbarrier, 3-stage slab pipeline), so the FP64 pipe is fed while
//     the next slab streams from L2;
//   * the epilogue is the whole trajectory state machine: norm test, descend / accept,
//     jump record, renormalisation, channel choice, threshold redraw, time bookkeeping,
//     period and dump accounting, the observables, and re-bucketing for the next step.
// FP64 has no tcgen05 kind, so the contraction runs on the FP64 FMA pipe; it is written
// so that every output keeps the oracle's k-ascending fma chain (bit-identical results).
#include "qjx_device.cuh"

namespace qjx {

constexpr long long kWaitLimit = 1ll << 24;  // bounded mbarrier polls before giving up

__device__ __forceinline__ double2 *slot_ptr(const Params &P, int slot, int tr)
{
    return P.psi + ((size_t)slot * P.n + tr) * P.MD;
}

__device__ __forceinline__ int group_of(const Params &P, const TrajState &s)
{
    switch (s.phase) {
    case PH_STEP: return s.b * P.deep + s.lvl;
    case PH_REC_W:
    case PH_REC_A: return P.gL0 + s.sub;
    case PH_OBS_E: return P.gHE;
    case PH_OBS_R: return P.gR0 + s.sub;
    default: return -1;
    }
}

__device__ __forceinline__ void enqueue(const Params &P, int *cnt, int *list, int g, int tr)
{
    const int pos = atomicAdd(&cnt[g], 1);
    list[(size_t)g * P.n + pos] = tr;
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
// Returns true when the last branch of a period finished.
__device__ __forceinline__ bool advance(TrajState &s, const double *dt, int nb)
{
    int l = s.lvl;
    unsigned long long m = s.mask;
    while (true) {
        if (!((m >> l) & 1ull)) {
            m |= (1ull << l);
            s.lvl = l;
            s.mask = m;
            return false;
        }
        m &= ~(1ull << l);
        if (l == 0) {
            s.mask = m;
            s.lvl = 0;
            s.b += 1;
            if (s.b == nb) {
                s.b = 0;
                return true;
            }
            return false;
        }
        l -= 1;
        s.t = __dadd_rn(__dsub_rn(s.t, dt[l]), dt[l]);
    }
}

// Observables of the state held in `col` (calc_chars_std[_start], core.cpp:665-725) and
// the normalised state psi / sqrt(norm) written to the spare slot for the energy and
// random-observable micro-steps.  Warp-cooperative; every lane computes the sequential
// sums identically.
__device__ void obs_prep(const Params &P, const TrajState &s, int tr, const double2 *col, double *wscr,
                         int lane, int dump, int is_start)
{
    const int d = P.d;
    const double nrm = seq_norm(col, d);
    const double sq = __dsqrt_rn(nrm);
    const double inv = __ddiv_rn(1.0, nrm);
    double2 *hat = slot_ptr(P, s.cur ^ 1, tr);
    double *adr_out = !P.o_adr ? nullptr
                      : (P.keep_adr ? P.o_adr + ((size_t)dump * P.n + tr) * d : P.o_adr + (size_t)tr * d);
    for (int k = lane; k < d; k += 32) {
        const double2 v = col[k];
        hat[k] = make_double2(__ddiv_rn(v.x, sq), __ddiv_rn(v.y, sq));
        const double a = __dmul_rn(__dadd_rn(0.0, __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y))), inv);
        wscr[k] = a;
        if (adr_out) adr_out[k] = a;
    }
    __syncwarp();
    double mean = 0.0;
    for (int k = 0; k < d; k++) mean = __dadd_rn(mean, __dmul_rn((double)k, wscr[k]));
    const double ms = is_start ? mean : P.mean_start[tr];
    const double disp = __dmul_rn(__dsub_rn(mean, ms), __dsub_rn(mean, ms));
    double m2 = 0.0;
    for (int k = 0; k < d; k++) {
        const double dk = __dsub_rn((double)k, mean);
        m2 = __dadd_rn(m2, __dmul_rn(__dmul_rn(dk, dk), wscr[k]));
    }
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
__device__ int after_step(const Params &P, TrajState &s, int tr, const double2 *col, double *wscr, int lane)
{
    if (advance(s, P.dt, P.nb)) {
        s.pc += 1;
        if (s.di < P.n_dumps && s.pc == P.dump_at[s.di]) {
            obs_prep(P, s, tr, col, wscr, lane, P.dump_base + s.di, 0);
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
    if (s.pc >= P.target) {
        s.phase = PH_DONE;
        return -1;
    }
    s.phase = PH_STEP;
    return s.b * P.deep + s.lvl;
}

// Apply the chosen jump channel: psi = (L_idx psi_hat) / sqrt(w_idx / g_idx)
// (experiment.cpp:1346-1369), record the channel, redraw eta (qj_proc.cpp:310-314) and
// count the finest-level step.
__device__ int apply_jump(const Params &P, TrajState &s, int tr, double2 *col, double *wscr, int lane, int idx,
                          double w_idx, int *err)
{
    const int d = P.d;
    const double q = __dsqrt_rn(__ddiv_rn(w_idx, P.g[idx]));
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
    s.phase = PH_STEP;
    s.t = __dadd_rn(s.t, P.dt[P.deep - 1]);
    return after_step(P, s, tr, col, wscr, lane);
}

// Warp-cooperative epilogue of one trajectory column: `col` holds M_g * psi in shared memory.
__device__ void column_epilogue(const Params &P, double2 *col, double2 *wscr_c, int tr, int *cnt_next,
                                int *list_next, int lane)
{
    const int d = P.d;
    double *wscr = reinterpret_cast<double *>(wscr_c);
    TrajState s = P.st[tr];
    int g2 = -1;
    int err = 0;
    bool paused = false;

    switch (s.phase) {
    case PH_STEP: {
        const double nrm = seq_norm(col, d);
        if (nrm > 1.0) {  // is_norm_crossed throws (experiment.cpp:1247-1251)
            err = ERR_NORM;
            break;
        }
        const double dt = P.dt[s.lvl];
        if (nrm > s.eta) {  // not crossed: accept psi' (qj_proc.cpp:317, 335)
            double2 *dst = slot_ptr(P, s.cur ^ 1, tr);
            for (int k = lane; k < d; k += 32) dst[k] = col[k];
            s.cur ^= 1;
            s.t = __dadd_rn(s.t, dt);
            g2 = after_step(P, s, tr, col, wscr, lane);
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
        double w = seq_norm(col, d);
        w = __dmul_rn(w, P.g[s.sub]);
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
            g2 = apply_jump(P, s, tr, col, wscr, lane, index, w, &err);
        } else {
            s.phase = PH_REC_A;
            s.sub = index;
            g2 = P.gL0 + index;
        }
    } break;

    case PH_REC_A: {
        const double w = P.gn[(size_t)tr * P.nd + s.sub];
        g2 = apply_jump(P, s, tr, col, wscr, lane, s.sub, w, &err);
    } break;

    case PH_OBS_E: {  // energy <psi_hat| H + E0 Hd |psi_hat>  (experiment.cpp:1423-1469)
        const double2 *hat = slot_ptr(P, s.cur ^ 1, tr);
        for (int k = lane; k < d; k += 32) wscr_c[k] = hat[k];
        __syncwarp();
        double e = 0.0;
        for (int k = 0; k < d; k++) {
            const double2 h = wscr_c[k], m = col[k];
            e = __dadd_rn(e, __dadd_rn(__dmul_rn(h.x, m.x), __dmul_rn(h.y, m.y)));
        }
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
        for (int k = lane; k < d; k += 32) wscr_c[k] = hat[k];
        __syncwarp();
        double rr = 0.0, ri = 0.0;
        for (int k = 0; k < d; k++) {
            const double2 h = wscr_c[k], m = col[k];
            const double cr = h.x, ci = -h.y;
            rr = __dadd_rn(rr, __dsub_rn(__dmul_rn(cr, m.x), __dmul_rn(ci, m.y)));
            ri = __dadd_rn(ri, __dadd_rn(__dmul_rn(ci, m.x), __dmul_rn(cr, m.y)));
        }
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

    if (lane == 0) {
        if (err) {
            s.err = err;
            s.phase = PH_ERROR;
            report_error(P, tr, err);
        } else if (paused) {
            s.paused = 1;
            atomicAdd(&P.ctrl[2], 1);
        } else if (g2 >= 0) {
            enqueue(P, cnt_next, list_next, g2, tr);
        }
        P.st[tr] = s;
    }
    __syncwarp();
}

// One lock-step micro-step: grouped FP64 GEMM over the buckets of step `s` (persistent
// CTAs stride over tiles) with the fused epilogue.  MD = 32 * MT padded rows.
template <int MT>
__global__ void __launch_bounds__(kThreads, 1) step_kernel(const Params P, int s)
{
    constexpr int MD = 32 * MT;
    constexpr int S16 = MD + 1;  // odd column stride: conflict-free column reads
    extern __shared__ __align__(128) unsigned char smem[];
    double2 *Bt = reinterpret_cast<double2 *>(smem);
    double2 *Us = Bt + kNC * S16;
    __shared__ __align__(8) uint64_t bar[kStages + 1];
    __shared__ int s_tstart[kMaxGroups + 1];
    __shared__ int s_tr[kNC];
    __shared__ long long s_src[kNC];
    __shared__ int s_abort;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ty = warp * 4 + (lane & 3), tx = lane >> 2;
    const int G = P.G, n = P.n, d = P.d;
    const int *cnt_cur = P.cnt + (s % 3) * G;
    int *cnt_next = P.cnt + ((s + 1) % 3) * G;
    const int *list_cur = P.lists + (size_t)(s & 1) * G * n;
    int *list_next = P.lists + (size_t)((s + 1) & 1) * G * n;

    if (blockIdx.x == 0)
        for (int i = tid; i < G; i += kThreads) P.cnt[((s + 2) % 3) * G + i] = 0;
    if (tid == 0) {
        int acc = 0;
        for (int g = 0; g < G; g++) {
            s_tstart[g] = acc;
            acc += (cnt_cur[g] + kNC - 1) / kNC;
        }
        s_tstart[G] = acc;
        for (int q = 0; q <= kStages; q++) mbar_init(&bar[q], 1);
        s_abort = 0;
    }
    __syncthreads();
    const int total = s_tstart[G];
    const int nslab = (d + kKB - 1) / kKB;
    uint32_t phase = 0;
    long long work = 0;

    for (int tile = blockIdx.x; tile < total; tile += gridDim.x) {
        int lo = 0, hi = G;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_tstart[mid] <= tile) lo = mid;
            else hi = mid;
        }
        const int g = lo;
        const int col0 = (tile - s_tstart[g]) * kNC;
        const int ncol = min(kNC, cnt_cur[g] - col0);
        if (tid < kNC) {
            if (tid < ncol) {
                const int tr = list_cur[(size_t)g * n + col0 + tid];
                const int ph = P.st[tr].phase, cur = P.st[tr].cur;
                const int slot = (ph >= PH_OBS_E) ? (cur ^ 1) : cur;
                s_tr[tid] = tr;
                s_src[tid] = ((long long)slot * n + tr) * MD;
            } else {
                s_tr[tid] = -1;
            }
        }
        __syncthreads();
        const double2 *mat = P.mats + (size_t)g * d * MD;
        if (tid == 0) {
            fence_proxy_async();
            mbar_expect_tx(&bar[kStages], (uint32_t)(ncol * d * 16));
            for (int c = 0; c < ncol; c++) bulk_g2s(Bt + c * S16, P.psi + s_src[c], (uint32_t)(d * 16), &bar[kStages]);
            for (int q = 0; q < kStages && q < nslab; q++) {
                const int kc = min(kKB, d - q * kKB);
                mbar_expect_tx(&bar[q], (uint32_t)(kc * MD * 16));
                bulk_g2s(Us + q * kKB * MD, mat + (size_t)q * kKB * MD, (uint32_t)(kc * MD * 16), &bar[q]);
            }
        }

        double2 acc[MT][kNT];
#pragma unroll
        for (int i = 0; i < MT; i++)
#pragma unroll
            for (int j = 0; j < kNT; j++) acc[i][j] = make_double2(0.0, 0.0);

        if (!mbar_wait_bounded(&bar[kStages], (phase >> kStages) & 1u, kWaitLimit)) s_abort = 1;
        phase ^= 1u << kStages;

        for (int sl = 0; sl < nslab; sl++) {
            const int q = sl % kStages;
            if (!mbar_wait_bounded(&bar[q], (phase >> q) & 1u, kWaitLimit)) s_abort = 1;
            phase ^= 1u << q;
            const int k0 = sl * kKB;
            const int kc = min(kKB, d - k0);
            const double2 *Uq = Us + q * kKB * MD;
            if (kc == kKB) {
#pragma unroll
                for (int kk = 0; kk < kKB; kk++) {
                    double2 a[MT], b[kNT];
#pragma unroll
                    for (int i = 0; i < MT; i++) a[i] = Uq[kk * MD + ty + 32 * i];
#pragma unroll
                    for (int j = 0; j < kNT; j++) b[j] = Bt[(tx + kTX * j) * S16 + k0 + kk];
#pragma unroll
                    for (int i = 0; i < MT; i++)
#pragma unroll
                        for (int j = 0; j < kNT; j++) {
                            acc[i][j].x = __fma_rn(a[i].x, b[j].x, acc[i][j].x);
                            acc[i][j].x = __fma_rn(-a[i].y, b[j].y, acc[i][j].x);
                            acc[i][j].y = __fma_rn(a[i].x, b[j].y, acc[i][j].y);
                            acc[i][j].y = __fma_rn(a[i].y, b[j].x, acc[i][j].y);
                        }
                }
            } else {
                for (int kk = 0; kk < kc; kk++) {
                    double2 a[MT], b[kNT];
#pragma unroll
                    for (int i = 0; i < MT; i++) a[i] = Uq[kk * MD + ty + 32 * i];
#pragma unroll
                    for (int j = 0; j < kNT; j++) b[j] = Bt[(tx + kTX * j) * S16 + k0 + kk];
#pragma unroll
                    for (int i = 0; i < MT; i++)
#pragma unroll
                        for (int j = 0; j < kNT; j++) {
                            acc[i][j].x = __fma_rn(a[i].x, b[j].x, acc[i][j].x);
                            acc[i][j].x = __fma_rn(-a[i].y, b[j].y, acc[i][j].x);
                            acc[i][j].y = __fma_rn(a[i].x, b[j].y, acc[i][j].y);
                            acc[i][j].y = __fma_rn(a[i].y, b[j].x, acc[i][j].y);
                        }
                }
            }
            __syncthreads();
            if (s_abort) break;
            if (tid == 0 && sl + kStages < nslab) {
                const int sn = sl + kStages;
                const int kn = min(kKB, d - sn * kKB);
                fence_proxy_async();
                mbar_expect_tx(&bar[q], (uint32_t)(kn * MD * 16));
                bulk_g2s(Us + q * kKB * MD, mat + (size_t)sn * kKB * MD, (uint32_t)(kn * MD * 16), &bar[q]);
            }
        }
        __syncthreads();
        if (s_abort) {
            if (tid == 0) {
                atomicAdd(&P.ctrl[4], 1);
                report_error(P, -1, ERR_TIMEOUT);
            }
            return;
        }

        // stage M_g * psi for the column-wise epilogue
#pragma unroll
        for (int i = 0; i < MT; i++) {
            const int row = ty + 32 * i;
            if (row < d) {
#pragma unroll
                for (int j = 0; j < kNT; j++) Bt[(tx + kTX * j) * S16 + row] = acc[i][j];
            }
        }
        __syncthreads();
        double2 *wscr = Us + warp * MD;
        for (int c = warp; c < ncol; c += kThreads / 32)
            column_epilogue(P, Bt + c * S16, wscr, s_tr[c], cnt_next, list_next, lane);
        work += ncol;
        fence_proxy_async();
        __syncthreads();
    }
    if (tid == 0 && work) atomicAdd((unsigned long long *)P.work, (unsigned long long)work);
}

// Bucket trajectories for step 0 of a call.  mode 0: start of a run of P.target periods;
// mode 1: resume trajectories paused on a full record buffer.
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
        s.paused = 0;
        s.phase = (P.target > 0) ? PH_STEP : PH_DONE;
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
    if (tr >= P.n) return;
    double2 *col = reinterpret_cast<double2 *>(smem) + (size_t)warp * 2 * P.MD;
    double *wscr = reinterpret_cast<double *>(col + P.MD);
    TrajState s = P.st[tr];
    if (s.phase == PH_ERROR) return;
    const double2 *src = slot_ptr(P, s.cur, tr);
    for (int k = lane; k < P.d; k += 32) col[k] = src[k];
    __syncwarp();
    obs_prep(P, s, tr, col, wscr, lane, dump, is_start);
    if (lane == 0) {
        s.pc = 0;
        s.di = 0;
        s.phase = PH_OBS_E;
        enqueue(P, P.cnt, P.lists, P.gHE, tr);
        P.st[tr] = s;
    }
}

__global__ void init_state_kernel(const Params P)
{
    const int tr = blockIdx.x * blockDim.x + threadIdx.x;
    if (tr >= P.n) return;
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
    s.pad = 0;
    P.st[tr] = s;
}

// eta_0 draw of trans_process_single (experiment.cpp:3260-3265)
__global__ void thresholds_kernel(const Params P)
{
    const int tr = blockIdx.x * blockDim.x + threadIdx.x;
    if (tr >= P.n) return;
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
template <int MT>
static cudaError_t launch_step_mt(const Params &P, int s, int grid, cudaStream_t st)
{
    constexpr int MD = 32 * MT;
    const size_t smem = (size_t)(kNC * (MD + 1) + kStages * kKB * MD) * sizeof(double2);
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(step_kernel<MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    step_kernel<MT><<<grid, kThreads, smem, st>>>(P, s);
    return cudaGetLastError();
}

cudaError_t launch_step(const Params &P, int s, int grid, cudaStream_t st)
{
    switch (P.MD / 32) {
    case 1: return launch_step_mt<1>(P, s, grid, st);
    case 2: return launch_step_mt<2>(P, s, grid, st);
    case 3: return launch_step_mt<3>(P, s, grid, st);
    case 4: return launch_step_mt<4>(P, s, grid, st);
    case 5: return launch_step_mt<5>(P, s, grid, st);
    case 6: return launch_step_mt<6>(P, s, grid, st);
    case 7: return launch_step_mt<7>(P, s, grid, st);
    case 8: return launch_step_mt<8>(P, s, grid, st);
    default: return cudaErrorInvalidValue;
    }
}

size_t step_smem_bytes(int MD) { return (size_t)(kNC * (MD + 1) + kStages * kKB * MD) * sizeof(double2); }

cudaError_t launch_schedule(const Params &P, int mode, cudaStream_t st)
{
    schedule_kernel<<<(P.n + 255) / 256, 256, 0, st>>>(P, mode);
    return cudaGetLastError();
}

cudaError_t launch_observe(const Params &P, int dump, int is_start, cudaStream_t st)
{
    const size_t smem = (size_t)8 * 2 * P.MD * sizeof(double2);
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(observe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)(8 * 2 * 32 * kMaxMT * sizeof(double2)));
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    observe_kernel<<<(P.n + 7) / 8, 256, smem, st>>>(P, dump, is_start);
    return cudaGetLastError();
}

cudaError_t launch_init_state(const Params &P, cudaStream_t st)
{
    init_state_kernel<<<(P.n + 255) / 256, 256, 0, st>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_thresholds(const Params &P, cudaStream_t st)
{
    thresholds_kernel<<<(P.n + 255) / 256, 256, 0, st>>>(P);
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

}  // namespace qjx
