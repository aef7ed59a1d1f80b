// qjx_lpn.cu -- Lyapunov paired trajectories (task_id 7, LpnMult) on the engine's states.
//
// Trajectories [0, n/2) are the bases and n/2 + b is the variation of base b.  After the
// bases' transient periods, lpn_kernel(mode 0) copies every base into its variation (psi, eta
// and the jump stream: copy_trajectory_lpn, experiment.cpp:2221-2244) and perturbs it
// (var_trajectory_lpn, experiment.cpp:2278-2397).  After every observation period,
// lpn_kernel(mode 1) takes the bases' characteristics (calc_chars_lpn, core.cpp:764-785) and
// runs lambda_lpn / lambda_lpn_now (experiment.cpp:3065-3135) for the variations: delta_f from
// their period-end characteristics, and when it leaves [delta_f_low, max(delta_f_high,
// 10 delta_s)] the log growth is added to lambda, the variation takes the base's current jump
// stream and eta (copy_stream_lpn) and is perturbed afresh around the base.
//
// One CTA per pair.  The pair's work is a handful of d x d complex matvecs (characteristics)
// plus one per bisection step of a renormalisation, thread per row, reading the FP64 matrices
// in the engine's transposed layout mats[g][k][row] (coalesced across the CTA's threads, L2
// resident across CTAs); next to the period's micro-steps this is a small cost.
//
// Arithmetic: every operation is the one the CPU oracle (lpn_oracle.c) performs: the canonical
// 32-lane sums of warp 0, k-ascending fma matvecs, and lpn_exp10 / lpn_log written out below
// from the mathematics (not the CUDA math library), so the variations' states, delta_s and
// lambda are bit-identical to the oracle's.
#include "qjx_device.cuh"

namespace qjx {

__device__ __forceinline__ double2 *lpn_slot(const Params &P, int slot, int tr)
{
    return P.psi + ((size_t)slot * P.n + tr) * P.MD;
}

// ---------------------------------------------------------------- exp10 / log
// exp10: Cody-Waite reduction x ln10 = k ln2 + r (x ln10 carried as p + q through an fma error
// term, ln2 as a 32-bit head and a tail), Taylor series of exp(r) to degree 16 in Horner form,
// times 2^k built from the exponent bits.  log: x = m 2^e, m in [sqrt(1/2), sqrt(2)),
// log m = 2 atanh(s) with s = (m - 1) / (m + 1) as a series in s^2 to s^25, plus e ln2.
__constant__ double kInvFact[17] = {
    0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p-1, 0x1.5555555555555p-3,
    0x1.5555555555555p-5, 0x1.1111111111111p-7, 0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-13,
    0x1.a01a01a01a01ap-16, 0x1.71de3a556c734p-19, 0x1.27e4fb7789f5cp-22, 0x1.ae64567f544e4p-26,
    0x1.1eed8eff8d898p-29, 0x1.6124613a86d09p-33, 0x1.93974a8c07c9dp-37, 0x1.ae7f3e733b81fp-41,
    0x1.ae7f3e733b81fp-45};
__constant__ double kInvOdd[13] = {
    0x1.0000000000000p+0, 0x1.5555555555555p-2, 0x1.999999999999ap-3, 0x1.2492492492492p-3,
    0x1.c71c71c71c71cp-4, 0x1.745d1745d1746p-4, 0x1.3b13b13b13b14p-4, 0x1.1111111111111p-4,
    0x1.e1e1e1e1e1e1ep-5, 0x1.af286bca1af28p-5, 0x1.8618618618618p-5, 0x1.642c8590b2164p-5,
    0x1.47ae147ae147bp-5};
constexpr double kLn2Hi = 0x1.62e42fee00000p-1, kLn2Lo = 0x1.a39ef35793c76p-33;
constexpr double kLn10Hi = 0x1.26bb1bbb55516p+1, kLn10Lo = -0x1.f48ad494ea3e9p-53;
constexpr double kLog2of10 = 0x1.a934f0979a371p+1;
constexpr double kSqrt2 = 0x1.6a09e667f3bcdp+0;

__device__ double lpn_exp10(double x)
{
    if (x != x) return x;
    if (x > 307.0) return __longlong_as_double(0x7ff0000000000000LL);
    if (x < -307.0) return 0.0;
    const double k = rint(__dmul_rn(x, kLog2of10));
    const double p = __dmul_rn(x, kLn10Hi);
    const double q = __fma_rn(x, kLn10Lo, __fma_rn(x, kLn10Hi, -p));
    const double r = __dadd_rn(__dsub_rn(p, __dmul_rn(k, kLn2Hi)), __dsub_rn(q, __dmul_rn(k, kLn2Lo)));
    double e = kInvFact[16];
    for (int n = 15; n >= 0; n--) e = __fma_rn(e, r, kInvFact[n]);
    return __dmul_rn(e, __longlong_as_double(((long long)k + 1023) << 52));
}

__device__ double lpn_log(double x)
{
    if (x != x || x < 0.0) return __longlong_as_double(0x7ff8000000000000LL);
    if (x == 0.0) return __longlong_as_double((long long)0xfff0000000000000ULL);
    if (x == __longlong_as_double(0x7ff0000000000000LL)) return x;
    double e = 0.0;
    unsigned long long b = (unsigned long long)__double_as_longlong(x);
    if ((b >> 52) == 0) {  // subnormal: scale by 2^54
        x = __dmul_rn(x, 0x1p54);
        b = (unsigned long long)__double_as_longlong(x);
        e = -54.0;
    }
    e = __dadd_rn(e, (double)((int)(b >> 52) - 1023));
    double m = __longlong_as_double((long long)((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL));
    if (m > kSqrt2) {
        m = __dmul_rn(m, 0.5);
        e = __dadd_rn(e, 1.0);
    }
    const double s = __ddiv_rn(__dsub_rn(m, 1.0), __dadd_rn(m, 1.0));
    const double z = __dmul_rn(s, s);
    double poly = kInvOdd[12];
    for (int k = 11; k >= 1; k--) poly = __fma_rn(poly, z, kInvOdd[k]);
    const double t = __dadd_rn(s, s);
    const double lm = __fma_rn(__dmul_rn(t, z), poly, t);
    return __dadd_rn(__dmul_rn(e, kLn2Hi), __dadd_rn(__dmul_rn(e, kLn2Lo), lm));
}

// ---------------------------------------------------------------- pair kernel
constexpr int kLpnThreads = 256;
constexpr int kLpnMaxRobs = 64;
enum { CH_MEAN = 1, CH_ENERGY = 2, CH_ROBS_ALL = 4 };

struct LpnChars {
    double mean, energy;
    double2 robs[kLpnMaxRobs];
};

struct LpnShared {
    LpnChars bc, vc;
    double red[4];  // [0] norm of the state under study, [1] |w|^2, [2] |base|^2
    double occ[24];  // MBL: cell occupations of the state under study
};

// The pair's ensemble: dimension, padded rows of its matrices, first group and the offset from a
// trajectory index to its Philox stream.
struct EnsCtx {
    int d, MD, g0;
    long long sbase;
};

__device__ __forceinline__ void cta_matvec(const Params &P, const EnsCtx &E, int g, const double2 *x, double2 *y)
{
    const int d = E.d, MD = E.MD;
    const double2 *mat = P.mats + P.g_off[E.g0 + g];
    for (int r = threadIdx.x; r < d; r += blockDim.x) {
        double re = 0.0, im = 0.0;
        for (int k = 0; k < d; k++) {
            const double2 m = mat[(size_t)k * MD + r];
            const double2 v = x[k];
            re = __fma_rn(m.x, v.x, re);
            re = __fma_rn(-m.y, v.y, re);
            im = __fma_rn(m.x, v.y, im);
            im = __fma_rn(m.y, v.x, im);
        }
        y[r] = make_double2(re, im);
    }
}

// calc_chars_lpn / calc_chars_std of `phi` (core.cpp:697-785) for the parts in `want` (robs_one
// >= 0: that random observable only) into `c`; the canonical norm is left in sh.red[0] and, with
// CH_MEAN, |phi_i|^2 / |phi|^2 in adr.  With MBL characteristics the mean is the imbalance
// (MBLCoreBehaviour::calc_chars_lpn, core.cpp:4753-4775; get_imbalance_mbl,
// experiment.cpp:1753-1800): one thread per cell sums its occupation over the basis words in
// order.  Ends with a barrier, so every thread may read `c` afterwards.
__device__ void cta_chars(const Params &P, const LpnParams &L, const EnsCtx &E, const double2 *phi, int want,
                          int robs_one, double2 *xh, double2 *y, LpnShared &sh, LpnChars &c, double *adr)
{
    const int d = E.d, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp == 0) {
        const double nrm = warp_norm(phi, d, lane);
        if (lane == 0) sh.red[0] = nrm;
        if (want & CH_MEAN) {
            const double inv = __ddiv_rn(1.0, nrm);
            double ms = 0.0;
            for (int st = lane; st < d; st += 32) {
                const double2 v = phi[st];
                const double a = __dmul_rn(__dadd_rn(0.0, __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y))), inv);
                adr[st] = a;
                ms = __dadd_rn(ms, __dmul_rn((double)st, a));
            }
            ms = warp_allsum(ms);
            if (lane == 0) c.mean = ms;
        }
    }
    __syncthreads();
    if ((want & CH_MEAN) && L.mbl_Nc > 0) {
        const int Nc = L.mbl_Nc;
        if ((int)threadIdx.x < Nc) {
            const int sh_bits = Nc - 1 - (int)threadIdx.x;  // cell c is bit Nc-1-c of a word
            double o = 0.0;
            for (int st = 0; st < d; st++) o = __dadd_rn(o, __dmul_rn(adr[st], (double)((L.words[st] >> sh_bits) & 1)));
            sh.occ[threadIdx.x] = o;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double even = 0.0, odd = 0.0;
            for (int cc = 0; cc < Nc; cc++) {
                if (cc % 2 == 0) even = __dadd_rn(even, sh.occ[cc]);
                else odd = __dadd_rn(odd, sh.occ[cc]);
            }
            c.mean = __ddiv_rn(__dsub_rn(even, odd), __dadd_rn(odd, even));
        }
        __syncthreads();
    }
    if (!(want & (CH_ENERGY | CH_ROBS_ALL)) && robs_one < 0) return;
    const double sq = __dsqrt_rn(sh.red[0]);
    for (int st = threadIdx.x; st < d; st += blockDim.x) {
        const double2 v = phi[st];
        xh[st] = make_double2(__ddiv_rn(v.x, sq), __ddiv_rn(v.y, sq));
    }
    __syncthreads();
    if (want & CH_ENERGY) {
        cta_matvec(P, E, P.gHE, xh, y);
        __syncthreads();
        if (warp == 0) {
            double es = 0.0;
            for (int st = lane; st < d; st += 32) {
                const double2 a = xh[st], b = y[st];
                es = __dadd_rn(es, __dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)));
            }
            es = warp_allsum(es);
            if (lane == 0) c.energy = es;
        }
        __syncthreads();
    }
    for (int o = 0; o < P.nr; o++) {
        if (!(want & CH_ROBS_ALL) && o != robs_one) continue;
        cta_matvec(P, E, P.gR0 + o, xh, y);
        __syncthreads();
        if (warp == 0) {
            double pr = 0.0, pi = 0.0;
            for (int st = lane; st < d; st += 32) {
                const double cr = xh[st].x, ci = -xh[st].y;
                const double2 b = y[st];
                pr = __dadd_rn(pr, __dsub_rn(__dmul_rn(cr, b.x), __dmul_rn(ci, b.y)));
                pi = __dadd_rn(pi, __dadd_rn(__dmul_rn(ci, b.x), __dmul_rn(cr, b.y)));
            }
            pr = warp_allsum(pr);
            pi = warp_allsum(pi);
            if (lane == 0) c.robs[o] = make_double2(pr, pi);
        }
        __syncthreads();
    }
}

// What calc_delta_s / calc_delta_f need of a state: CH_ parts and one random-observable slot
// (-1: none).  MBL: -1 the spec (slot 0), -2 the imbalance, k >= 0 slot k + 1; JCS: -1 the spec
// (slot 0), -2 <a^+ a> (the energy observable), k >= 0 slot k + 1; Integrable: -1 the spec (slot
// 0), k >= 0 slot k + 1.
__device__ __forceinline__ bool spec_sys(const LpnParams &L) { return L.chars_sys != 0; }

__device__ __forceinline__ int delta_want(const LpnParams &L)
{
    if (L.mbl_Nc > 0) return L.lpn_type == -2 ? CH_MEAN : 0;
    if (L.chars_sys == 1) return L.lpn_type == -2 ? CH_ENERGY : 0;
    if (L.chars_sys == 5) return 0;
    return L.lpn_type == -1 ? CH_MEAN : L.lpn_type == -2 ? CH_ENERGY : 0;
}

__device__ __forceinline__ int delta_one(const LpnParams &L)
{
    if (spec_sys(L)) return L.lpn_type == -1 ? 0 : L.lpn_type >= 0 ? L.lpn_type + 1 : -1;
    return L.lpn_type >= 0 ? L.lpn_type : -1;
}

// calc_delta_s / calc_delta_f (dimer core.cpp:839-901, JCS core.cpp:2870-2975, MBL
// core.cpp:4823-4901, Integrable core.cpp:6606-6676), variation v against base b
__device__ __forceinline__ double lpn_delta(const EnsCtx &E, const LpnParams &L, const LpnChars &v,
                                            const LpnChars &b)
{
    if (spec_sys(L) && L.lpn_type == -1) {  // spec = <H> / W or <a> / alpha, real divisions
        const double2 bb = b.robs[0], vv = v.robs[0];
        const double dr = __dsub_rn(__ddiv_rn(bb.x, L.spec_div), __ddiv_rn(vv.x, L.spec_div));
        const double di = __dsub_rn(__ddiv_rn(bb.y, L.spec_div), __ddiv_rn(vv.y, L.spec_div));
        return __dsqrt_rn(__dadd_rn(__dmul_rn(dr, dr), __dmul_rn(di, di)));
    }
    if (L.mbl_Nc > 0 && L.lpn_type == -2) return fabs(__dsub_rn(v.mean, b.mean));
    if (L.chars_sys == 1 && L.lpn_type == -2) return __ddiv_rn(fabs(__dsub_rn(v.energy, b.energy)), (double)E.d);
    if (L.lpn_type == -1) return __ddiv_rn(fabs(__dsub_rn(v.mean, b.mean)), (double)E.d);
    if (L.lpn_type == -2) return __ddiv_rn(fabs(__dsub_rn(v.energy, b.energy)), L.max_energy);
    const int o = delta_one(L);
    const double2 bb = b.robs[o], vv = v.robs[o];
    const double dr = __dsub_rn(bb.x, vv.x), di = __dsub_rn(bb.y, vv.y);
    return __dsqrt_rn(__dadd_rn(__dmul_rn(dr, dr), __dmul_rn(di, di)));
}

// var_trajectory_lpn (experiment.cpp:2278-2397) of variation v around the base state pb:
// a fresh direction w from the variation stream (uniforms 2u - 1, real parts then imaginary
// parts), |w| = 1, and eps = 10^m bisected in m until |delta_s - target| < eps_error or
// eps_deep halvings; a delta_s that is neither above nor below the target ends the search.
// Leaves the perturbed state in pv.
__device__ void var_trajectory(const Params &P, const EnsCtx &E, const LpnParams &L, int v, const double2 *pb,
                               double2 *pv, double2 *w, double2 *xh, double2 *y, LpnShared &sh, double *adr)
{
    const int d = E.d, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long pos0 = L.var_pos[v];
    const unsigned long long stream = (1ULL << 63) | (unsigned long long)(E.sbase + v);
    for (int st = threadIdx.x; st < d; st += blockDim.x) {
        const double ur = philox_uniform(777ULL, stream, (unsigned long long)(pos0 + st));
        const double ui = philox_uniform(777ULL, stream, (unsigned long long)(pos0 + d + st));
        w[st] = make_double2(__dsub_rn(__dmul_rn(2.0, ur), 1.0), __dsub_rn(__dmul_rn(2.0, ui), 1.0));
    }
    __syncthreads();
    if (warp == 0) {
        const double nw = warp_norm(w, d, lane);
        const double nb = warp_norm(pb, d, lane);
        if (lane == 0) {
            sh.red[1] = nw;
            sh.red[2] = nb;
        }
    }
    __syncthreads();
    const double sw = __dsqrt_rn(sh.red[1]);
    const double s2 = __dsqrt_rn(sh.red[2]);
    for (int st = threadIdx.x; st < d; st += blockDim.x) {
        const double2 a = w[st];
        w[st] = make_double2(__ddiv_rn(a.x, sw), __ddiv_rn(a.y, sw));
    }
    if (threadIdx.x == 0) L.var_pos[v] = pos0 + 2LL * d;
    double lo = L.eps_low, hi = L.eps_high, diff = __dsub_rn(hi, lo);
    int deep = 0;
    double eps = lpn_exp10(__dmul_rn(__dadd_rn(lo, hi), 0.5));
    const int want = delta_want(L), one = delta_one(L);
    __syncthreads();
    while (deep < L.eps_deep) {
        for (int st = threadIdx.x; st < d; st += blockDim.x) {
            const double2 a = pb[st], b = w[st];
            pv[st] = make_double2(__dadd_rn(a.x, __dmul_rn(eps, b.x)), __dadd_rn(a.y, __dmul_rn(eps, b.y)));
        }
        __syncthreads();
        if (warp == 0) {
            const double nm = warp_norm(pv, d, lane);
            if (lane == 0) sh.red[0] = nm;
        }
        __syncthreads();
        const double sm = __dsqrt_rn(sh.red[0]);
        for (int st = threadIdx.x; st < d; st += blockDim.x) {
            const double2 a = pv[st];
            pv[st] = make_double2(__dmul_rn(__ddiv_rn(a.x, sm), s2), __dmul_rn(__ddiv_rn(a.y, sm), s2));
        }
        __syncthreads();
        cta_chars(P, L, E, pv, want, one, xh, y, sh, sh.vc, adr);
        const double ds = lpn_delta(E, L, sh.vc, sh.bc);
        if (fabs(__dsub_rn(ds, L.delta_s)) < L.eps_error) break;
        if (ds > L.delta_s) {
            hi = __dsub_rn(hi, __dmul_rn(0.5, diff));
        } else if (ds < L.delta_s) {
            lo = __dadd_rn(lo, __dmul_rn(0.5, diff));
        } else {
            break;
        }
        diff = __dsub_rn(hi, lo);
        deep++;
        eps = lpn_exp10(__dmul_rn(__dadd_rn(lo, hi), 0.5));
        __syncthreads();  // every thread has read sh.vc before the next step rewrites it
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        L.eps_iters[v] = deep;
        L.eps[v] = eps;
    }
}

__device__ void store_chars(const Params &P, const LpnParams &L, int tr, const LpnChars &c)
{
    if (threadIdx.x == 0) {
        L.mean_lpn[tr] = L.chars_sys == 1 ? c.energy : c.mean;  // JCS: get_num_photons_jcs
        L.energy_lpn[tr] = c.energy;
    }
    for (int o = threadIdx.x; o < P.nr; o += blockDim.x) L.robs_lpn[(size_t)tr * P.nr + o] = c.robs[o];
}

// mode 0: start (after the bases' transient); mode 1: after one observation period at curr_time;
// mode 2: the bases' characteristics only (LpnMultDeep sub-periods between Lyapunov updates).
// adr_dump >= 0: the variations' |psi_i|^2 / |psi|^2 after the update go to that dump's adr slot.
__global__ void __launch_bounds__(kLpnThreads) lpn_kernel(const Params P, const LpnParams L, int mode,
                                                           double curr_time, int adr_dump)
{
    extern __shared__ __align__(16) unsigned char smem[];
    LpnShared &sh = *reinterpret_cast<LpnShared *>(smem);
    double2 *pb = reinterpret_cast<double2 *>(smem + ((sizeof(LpnShared) + 15) & ~(size_t)15));
    double2 *pv = pb + P.MD, *w = pv + P.MD, *xh = w + P.MD, *y = xh + P.MD;
    double *adr = reinterpret_cast<double *>(y + P.MD);
    // pair -> its ensemble e (pairs of ensemble e are pair0[e] .. pair0[e + 1] - 1): base b and
    // variation v = b + n_e / 2 of that ensemble
    int lo = 0, hi = P.E;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (L.pair0[mid] <= (int)blockIdx.x) lo = mid;
        else hi = mid;
    }
    const int t0 = P.e_tr0[lo], half = (P.e_tr0[lo + 1] - t0) / 2;
    const int b = t0 + (int)blockIdx.x - L.pair0[lo], v = b + half;
    const EnsCtx E{P.e_d[lo], 8 * ((P.e_d[lo] + 7) / 8), P.e_g0[lo], P.e_sbase[lo] - t0};
    const int d = E.d;
    const TrajState sb = P.st[b];
    TrajState sv = P.st[v];
    if (sb.phase == PH_ERROR || sv.phase == PH_ERROR) return;
    const double2 *gb = lpn_slot(P, sb.cur, b);
    double2 *gv = lpn_slot(P, sv.cur, v);
    for (int st = threadIdx.x; st < d; st += blockDim.x) {
        pb[st] = gb[st];
        pv[st] = gv[st];
    }
    __syncthreads();
    const int full = CH_MEAN | CH_ENERGY | CH_ROBS_ALL;
    cta_chars(P, L, E, pb, full, -1, xh, y, sh, sh.bc, adr);  // calc_chars_lpn of the base
    store_chars(P, L, b, sh.bc);
    if (mode == 2) return;
    bool moved = false;
    if (mode == 0) {
        // copy_trajectory_lpn + var_trajectory_lpn; calc_chars_lpn_start
        sv.rng_src = sb.rng_src;
        sv.rng_pos = sb.rng_pos;
        sv.eta = sb.eta;
        for (int st = threadIdx.x; st < d; st += blockDim.x) pv[st] = pb[st];
        __syncthreads();
        var_trajectory(P, E, L, v, pb, pv, w, xh, y, sh, adr);
        moved = true;
        cta_chars(P, L, E, pv, full, -1, xh, y, sh, sh.vc, adr);
        store_chars(P, L, v, sh.vc);
        if (threadIdx.x == 0) {
            L.delta_s_v[v] = lpn_delta(E, L, sh.vc, sh.bc);
            L.delta_s_v[b] = 0.0;
            L.lambda[b] = L.lambda[v] = 0.0;
            L.lambda_now[b] = L.lambda_now[v] = 0.0;
            L.num_renorms[b] = L.num_renorms[v] = 0;
            L.renormed[b] = L.renormed[v] = 0;
        }
    } else {
        const int want = delta_want(L), one = delta_one(L);
        cta_chars(P, L, E, pv, want, one, xh, y, sh, sh.vc, adr);
        const double df = lpn_delta(E, L, sh.vc, sh.bc);
        const double ds = L.delta_s_v[v];
        const double ds10 = __dmul_rn(ds, 10.0);
        const double lim = (L.delta_f_high < ds10) ? ds10 : L.delta_f_high;  // std::max
        __syncthreads();  // sh.vc is rewritten below
        if (L.per_period || df > lim || df < L.delta_f_low) {
            const double ratio = __ddiv_rn(df, ds);
            const double lam = __dadd_rn(L.lambda[v], lpn_log(__dadd_rn(ratio, 1.0e-16)));
            sv.rng_src = sb.rng_src;  // copy_stream_lpn
            sv.rng_pos = sb.rng_pos;
            sv.eta = sb.eta;
            var_trajectory(P, E, L, v, pb, pv, w, xh, y, sh, adr);
            moved = true;
            cta_chars(P, L, E, pv, full, -1, xh, y, sh, sh.vc, adr);
            store_chars(P, L, v, sh.vc);
            if (threadIdx.x == 0) {
                L.lambda[v] = lam;
                L.num_renorms[v] += 1;
                L.renormed[v] = 1;
                L.ratio[v] = ratio;
                L.ds_rec[v] = ds;
                L.df_rec[v] = df;
                L.delta_s_v[v] = lpn_delta(E, L, sh.vc, sh.bc);
                L.lambda_now[v] = __ddiv_rn(lam, curr_time);
            }
        } else {
            cta_chars(P, L, E, pv, full, -1, xh, y, sh, sh.vc, adr);
            store_chars(P, L, v, sh.vc);
            if (threadIdx.x == 0) {
                L.renormed[v] = 0;
                L.lambda_now[v] =
                    __ddiv_rn(__dadd_rn(L.lambda[v], lpn_log(__dadd_rn(__ddiv_rn(df, ds), 1.0e-16))), curr_time);
            }
        }
    }
    if (moved) {
        for (int st = threadIdx.x; st < d; st += blockDim.x) gv[st] = pv[st];
        if (threadIdx.x == 0) P.st[v] = sv;
    }
    if (adr_dump >= 0 && P.o_adr) {
        double *dst = P.keep_adr ? P.o_adr + ((size_t)adr_dump * P.n + v) * P.d : P.o_adr + (size_t)v * P.d;
        cta_chars(P, L, E, pv, CH_MEAN, -1, xh, y, sh, sh.vc, adr);
        for (int st = threadIdx.x; st < d; st += blockDim.x) dst[st] = adr[st];
    }
}

size_t lpn_smem_bytes(int MD)
{
    return ((sizeof(LpnShared) + 15) & ~(size_t)15) + 5 * (size_t)MD * sizeof(double2) + (size_t)MD * sizeof(double);
}

cudaError_t launch_lpn(const Params &P, const LpnParams &L, int mode, double curr_time, int adr_dump,
                       cudaStream_t st)
{
    const int pairs = L.pairs;
    if (pairs == 0) return cudaSuccess;
    const size_t smem = lpn_smem_bytes(P.MD);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(lpn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    lpn_kernel<<<pairs, kLpnThreads, smem, st>>>(P, L, mode, curr_time, adr_dump);
    return cudaGetLastError();
}

}  // namespace qjx
