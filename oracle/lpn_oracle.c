/*
 * lpn_oracle.c -- CPU restatement of the Lyapunov paired-trajectory task of QJX (task_id 7,
 * LpnMult) on top of the QJ restatement in qjx_oracle.c (TEST INFRASTRUCTURE: only tests/ load it).
 *
 *   LpnMult trans / obser   source/cpp/QJX/QJX/experiment.cpp:138-286
 *   copy_trajectory_lpn     experiment.cpp:2221-2244  (phi, eta and the jump stream of the base)
 *   copy_stream_lpn         experiment.cpp:2246-2256
 *   var_trajectory_lpn      experiment.cpp:2278-2397  (random direction, eps bisection in log10)
 *   lambda_lpn              experiment.cpp:3065-3105; lambda_lpn_now 3107-3135
 *   calc_chars_lpn[_start]  core.cpp:727-785; calc_delta_s / calc_delta_f core.cpp:839-901
 *   max_energy              newdel_exp.cpp:540-550 (passed in by the caller)
 *
 * Trajectories [0, n/2) are the bases, n/2 + b is the variation of base b.  The variation
 * stream (streams_var, MCG31 seed 777 leapfrogged per trajectory, newdel_exp.cpp:313-330) is
 * Philox4x32-10 under key 777 on stream 2^63 + tr_base + tr; its uniforms on [-1, 1] are
 * 2u - 1 with u in (0, 1].  pow(10, x) and log(x) are lpn_exp10 / lpn_log below, written
 * from the mathematics so that the CUDA engine evaluates the same operations; glibc's pow
 * and log agree with them to a few ulp (checked by the tests).
 *
 * Build: with qjx_oracle.c (oracle/build_oracle.py, -ffp-contract=off: only explicit fma fuses).
 */
#include "qjx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ exp10 / log
 * exp10: Cody-Waite reduction x ln10 = k ln2 + r, |r| <= ln2 / 2 (x ln10 carried as p + q by an
 * fma error term; ln2 split into a 32-bit head and a tail so k * LN2_HI is exact), then the Taylor
 * series of exp(r) to degree 16 in Horner form with fma, scaled by 2^k through the exponent bits.
 * log: x = m 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s), s = (m - 1) / (m + 1), series
 * in s^2 to s^25 in Horner form, plus e ln2 (head + tail). */
static const double LN2_HI = 0x1.62e42fee00000p-1, LN2_LO = 0x1.a39ef35793c76p-33;
static const double LN10_HI = 0x1.26bb1bbb55516p+1, LN10_LO = -0x1.f48ad494ea3e9p-53;
static const double LOG2_10 = 0x1.a934f0979a371p+1;
static const double SQRT2 = 0x1.6a09e667f3bcdp+0;
/* 1/n!, n = 0..16 */
static const double INV_FACT[17] = {
    0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p-1, 0x1.5555555555555p-3,
    0x1.5555555555555p-5, 0x1.1111111111111p-7, 0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-13,
    0x1.a01a01a01a01ap-16, 0x1.71de3a556c734p-19, 0x1.27e4fb7789f5cp-22, 0x1.ae64567f544e4p-26,
    0x1.1eed8eff8d898p-29, 0x1.6124613a86d09p-33, 0x1.93974a8c07c9dp-37, 0x1.ae7f3e733b81fp-41,
    0x1.ae7f3e733b81fp-45};
/* 1/(2k+1), k = 1..12 */
static const double INV_ODD[13] = {
    0x1.0000000000000p+0, 0x1.5555555555555p-2, 0x1.999999999999ap-3, 0x1.2492492492492p-3,
    0x1.c71c71c71c71cp-4, 0x1.745d1745d1746p-4, 0x1.3b13b13b13b14p-4, 0x1.1111111111111p-4,
    0x1.e1e1e1e1e1e1ep-5, 0x1.af286bca1af28p-5, 0x1.8618618618618p-5, 0x1.642c8590b2164p-5,
    0x1.47ae147ae147bp-5};

static double bits_double(uint64_t b)
{
    double x;
    memcpy(&x, &b, sizeof(x));
    return x;
}

static uint64_t double_bits(double x)
{
    uint64_t b;
    memcpy(&b, &x, sizeof(b));
    return b;
}

double orc_lpn_exp10(double x)
{
    if (x != x) return x;
    if (x > 307.0) return INFINITY;
    if (x < -307.0) return 0.0;
    const double k = rint(x * LOG2_10);
    const double p = x * LN10_HI;
    const double q = fma(x, LN10_LO, fma(x, LN10_HI, -p));
    const double r = (p - k * LN2_HI) + (q - k * LN2_LO);
    double e = INV_FACT[16];
    for (int n = 15; n >= 0; n--) e = fma(e, r, INV_FACT[n]);
    return e * bits_double((uint64_t)((int64_t)k + 1023) << 52);
}

double orc_lpn_log(double x)
{
    if (x != x || x < 0.0) return NAN;
    if (x == 0.0) return -INFINITY;
    if (x == INFINITY) return x;
    double e = 0.0;
    uint64_t b = double_bits(x);
    if ((b >> 52) == 0) {  /* subnormal: scale by 2^54 */
        x = x * 0x1p54;
        b = double_bits(x);
        e = -54.0;
    }
    e = e + (double)((int)(b >> 52) - 1023);
    double m = bits_double((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (m > SQRT2) {
        m = m * 0.5;
        e = e + 1.0;
    }
    const double s = (m - 1.0) / (m + 1.0);
    const double z = s * s;
    double poly = INV_ODD[12];
    for (int k = 11; k >= 1; k--) poly = fma(poly, z, INV_ODD[k]);
    const double t = s + s;
    const double lm = fma(t * z, poly, t);
    return e * LN2_HI + (e * LN2_LO + lm);
}

/* ------------------------------------------------------------------ characteristics */
static double lanes_sum(double p[32])
{
    for (int off = 16; off >= 1; off >>= 1) {
        double q[32];
        for (int l = 0; l < 32; l++) q[l] = p[l] + p[l ^ off];
        memcpy(p, q, sizeof(q));
    }
    return p[0];
}

enum { CH_MEAN = 1, CH_ENERGY = 2, CH_ROBS_ALL = 4 };

typedef struct {
    double mean, energy;
    double robs[2 * 64];
} chars_t;

/* MBL: the imbalance of an adr row (get_imbalance_mbl, experiment.cpp:1753-1800): cell
 * occupations summed over the basis words in order, then (even cells - odd cells) / all. */
static double mbl_imbalance_row(int Nc, int d, const int *words, const double *adr)
{
    double occ[32];
    for (int c = 0; c < Nc; c++) occ[c] = 0.0;
    for (int s = 0; s < d; s++)
        for (int c = 0; c < Nc; c++) occ[c] = occ[c] + adr[s] * (double)((words[s] >> (Nc - 1 - c)) & 1);
    double even = 0.0, odd = 0.0;
    for (int c = 0; c < Nc; c++) {
        if (c % 2 == 0) even = even + occ[c];
        else odd = odd + occ[c];
    }
    return (even - odd) / (odd + even);
}

/* calc_chars_lpn / calc_chars_std of one state (core.cpp:697-785): the operations of
 * orc_observables for the parts in `want`; `robs_one` >= 0 asks for that random observable only.
 * With MBL words (mbl_Nc > 0) the mean is the imbalance (MBLCoreBehaviour::calc_chars_lpn,
 * core.cpp:4753-4775). */
static void lpn_chars(const orc_problem *p, const double *phi, int want, int robs_one, double *xh, double *sm,
                      chars_t *c, int mbl_Nc, const int *words)
{
    const int d = p->d;
    const double norm = orc_norm_square(d, phi);
    if (want & CH_MEAN) {
        double ps[32] = {0};
        const double inv = 1.0 / norm;
        for (int st = 0; st < d; st++) {
            const double a = phi[2 * st] * phi[2 * st], b = phi[2 * st + 1] * phi[2 * st + 1];
            const double adr = (0.0 + (a + b)) * inv;
            ps[st & 31] = ps[st & 31] + (double)st * adr;
            sm[st] = adr;
        }
        c->mean = mbl_Nc > 0 ? mbl_imbalance_row(mbl_Nc, d, words, sm) : lanes_sum(ps);
    }
    if (!(want & (CH_ENERGY | CH_ROBS_ALL)) && robs_one < 0) return;
    const double sq = sqrt(norm);
    for (int st = 0; st < d; st++) {
        xh[2 * st] = phi[2 * st] / sq;
        xh[2 * st + 1] = phi[2 * st + 1] / sq;
    }
    if (want & CH_ENERGY) {
        orc_matvec(d, p->HE, xh, sm);
        double ps[32] = {0};
        for (int st = 0; st < d; st++) {
            const double a = xh[2 * st] * sm[2 * st], b = xh[2 * st + 1] * sm[2 * st + 1];
            ps[st & 31] = ps[st & 31] + (a + b);
        }
        c->energy = lanes_sum(ps);
    }
    for (int o = 0; o < p->num_robs; o++) {
        if (!(want & CH_ROBS_ALL) && o != robs_one) continue;
        orc_matvec(d, p->R + 2 * (size_t)o * d * d, xh, sm);
        double pr[32] = {0}, pi[32] = {0};
        for (int st = 0; st < d; st++) {
            const double cr = xh[2 * st], ci = -xh[2 * st + 1];
            pr[st & 31] = pr[st & 31] + (cr * sm[2 * st] - ci * sm[2 * st + 1]);
            pi[st & 31] = pi[st & 31] + (ci * sm[2 * st] + cr * sm[2 * st + 1]);
        }
        c->robs[2 * o] = lanes_sum(pr);
        c->robs[2 * o + 1] = lanes_sum(pi);
    }
}

/* what calc_delta_s / calc_delta_f need of a state: a CH_ part (delta_want) and / or one random
 * observable slot (delta_one, -1 none) */
static int spec_sys(const orc_lpn_config *cfg) { return cfg->chars_sys != 0; }

static int delta_want(const orc_lpn_config *cfg)
{
    if (cfg->mbl_Nc > 0) return cfg->lpn_type == -2 ? CH_MEAN : 0;
    if (cfg->chars_sys == 1) return cfg->lpn_type == -2 ? CH_ENERGY : 0;
    if (cfg->chars_sys == 5) return 0;
    return cfg->lpn_type == -1 ? CH_MEAN : cfg->lpn_type == -2 ? CH_ENERGY : 0;
}

static int delta_one(const orc_lpn_config *cfg)
{
    if (spec_sys(cfg)) return cfg->lpn_type == -1 ? 0 : cfg->lpn_type >= 0 ? cfg->lpn_type + 1 : -1;
    return cfg->lpn_type >= 0 ? cfg->lpn_type : -1;
}

/* calc_delta_s / calc_delta_f (dimer core.cpp:839-901; MBL core.cpp:4823-4901): var against base */
static double lpn_delta(const orc_problem *p, const orc_lpn_config *cfg, const chars_t *v, const chars_t *b)
{
    if (spec_sys(cfg) && cfg->lpn_type == -1) { /* spec = <H> / W or <a> / alpha, real divisions */
        const double dr = b->robs[0] / cfg->spec_div - v->robs[0] / cfg->spec_div;
        const double di = b->robs[1] / cfg->spec_div - v->robs[1] / cfg->spec_div;
        return sqrt(dr * dr + di * di);
    }
    if (cfg->mbl_Nc > 0 && cfg->lpn_type == -2) return fabs(v->mean - b->mean);
    if (cfg->chars_sys == 1 && cfg->lpn_type == -2) return fabs(v->energy - b->energy) / (double)p->d;
    if (cfg->lpn_type == -1) return fabs(v->mean - b->mean) / (double)p->d;
    if (cfg->lpn_type == -2) return fabs(v->energy - b->energy) / cfg->max_energy;
    const int o = delta_one(cfg);
    const double dr = b->robs[2 * o] - v->robs[2 * o], di = b->robs[2 * o + 1] - v->robs[2 * o + 1];
    return sqrt(dr * dr + di * di);
}

static int lpn_type_ok(const orc_problem *p, const orc_lpn_config *cfg)
{
    if (cfg->mbl_Nc > 0 && (orc_mbl_basis(cfg->mbl_Nc, NULL) != p->d || cfg->mbl_Nc > 24 || p->num_robs < 1))
        return 0;
    if (cfg->chars_sys != 0 && cfg->chars_sys != 1 && cfg->chars_sys != 3 && cfg->chars_sys != 5) return 0;
    if ((cfg->chars_sys == 3) != (cfg->mbl_Nc > 0)) return 0;
    if (cfg->chars_sys != 0 && p->num_robs < 1) return 0;
    if (cfg->chars_sys == 5 && cfg->lpn_type == -2) return 0;
    const int shift = spec_sys(cfg) ? 1 : 0;
    return cfg->lpn_type == -1 || cfg->lpn_type == -2 ||
           (cfg->lpn_type >= 0 && cfg->lpn_type + shift < p->num_robs);
}

/* the MBL basis words of cfg (NULL for the dimer); the caller frees */
static int *lpn_words(const orc_lpn_config *cfg)
{
    if (cfg->mbl_Nc <= 0) return NULL;
    int *w = (int *)malloc(sizeof(int) * (size_t)orc_mbl_basis(cfg->mbl_Nc, NULL));
    if (w) orc_mbl_basis(cfg->mbl_Nc, w);
    return w;
}

static double var_uniform(const orc_problem *p, int tr, int64_t *pos)
{
    const double u = orc_philox_uniform(777u, (1ULL << 63) | (p->tr_base + (uint64_t)tr), (uint64_t)(*pos)++);
    return 2.0 * u - 1.0;
}

/* var_trajectory_lpn (experiment.cpp:2278-2397): phi_v = sqrt(|base|^2) (base + eps w) / |base + eps w|
 * with a fresh random direction w, |w| = 1, and eps = 10^m bisected in m over [eps_low, eps_high]
 * until |delta_s - target| < eps_error or eps_deep halvings.  A delta_s that is neither above nor
 * below the target (NaN, or equal with eps_error <= 0) ends the search (the reference would not
 * terminate).  Returns the halvings done; *eps_out gets the last eps. */
static int var_trajectory(const orc_problem *p, const orc_lpn_config *cfg, orc_lpn *lp, const double *base_phi,
                          double *phi, int v, const chars_t *bc, double *w, double *xh, double *sm, double *eps_out,
                          const int *words)
{
    const int d = p->d;
    for (int st = 0; st < d; st++) w[2 * st] = var_uniform(p, v, &lp->var_pos[v]);
    for (int st = 0; st < d; st++) w[2 * st + 1] = var_uniform(p, v, &lp->var_pos[v]);
    const double nw = orc_norm_square(d, w);
    for (int st = 0; st < d; st++) {
        w[2 * st] = w[2 * st] / sqrt(nw);
        w[2 * st + 1] = w[2 * st + 1] / sqrt(nw);
    }
    const double norm_2 = orc_norm_square(d, base_phi);
    double lo = cfg->eps_low, hi = cfg->eps_high, diff = hi - lo;
    int deep = 0;
    double eps = orc_lpn_exp10((lo + hi) * 0.5);
    const int want = delta_want(cfg), one = delta_one(cfg);
    while (deep < cfg->eps_deep) {
        for (int st = 0; st < 2 * d; st++) phi[st] = base_phi[st] + eps * w[st];
        const double nm = orc_norm_square(d, phi);
        for (int st = 0; st < 2 * d; st++) phi[st] = phi[st] / sqrt(nm);
        for (int st = 0; st < 2 * d; st++) phi[st] = phi[st] * sqrt(norm_2);
        chars_t vc;
        lpn_chars(p, phi, want, one, xh, sm, &vc, cfg->mbl_Nc, words);
        const double ds = lpn_delta(p, cfg, &vc, bc);
        if (fabs(ds - cfg->delta_s) < cfg->eps_error) break;
        if (ds > cfg->delta_s) {
            hi = hi - 0.5 * diff;
        } else if (ds < cfg->delta_s) {
            lo = lo + 0.5 * diff;
        } else {
            break;
        }
        diff = hi - lo;
        deep++;
        eps = orc_lpn_exp10((lo + hi) * 0.5);
    }
    *eps_out = eps;
    return deep;
}

static void store_chars(const orc_problem *p, const orc_lpn_config *cfg, orc_lpn *lp, int tr, const chars_t *c)
{
    lp->mean_lpn[tr] = cfg->chars_sys == 1 ? c->energy : c->mean; /* JCS: get_num_photons_jcs */
    lp->energy_lpn[tr] = c->energy;
    for (int o = 0; o < p->num_robs; o++) {
        lp->robs_lpn[2 * ((size_t)tr * p->num_robs + o)] = c->robs[2 * o];
        lp->robs_lpn[2 * ((size_t)tr * p->num_robs + o) + 1] = c->robs[2 * o + 1];
    }
}

static void copy_stream(orc_state *s, int v, int b)
{
    s->rng_src[v] = s->rng_src[b];
    s->rng_pos[v] = s->rng_pos[b];
    s->eta[v] = s->eta[b];
}

int orc_lpn_start(const orc_problem *p, orc_state *s, const orc_lpn_config *cfg, orc_lpn *lp)
{
    const int d = p->d, n = p->n_traj, half = n / 2;
    if (!lpn_type_ok(p, cfg) || p->num_robs > 64 || !s->rng_src || (n & 1)) return 2;
    const int full = CH_MEAN | CH_ENERGY | CH_ROBS_ALL;
    int *words = lpn_words(cfg);
    if (cfg->mbl_Nc > 0 && !words) return 1;
    int bad = 0;
#pragma omp parallel
    {
        double *w = (double *)malloc(sizeof(double) * 2 * d);
        double *xh = (double *)malloc(sizeof(double) * 2 * d);
        double *sm = (double *)malloc(sizeof(double) * 2 * d);
        if (!w || !xh || !sm) {
#pragma omp atomic write
            bad = 1;
        } else {
#pragma omp for schedule(dynamic, 1)
            for (int b = 0; b < half; b++) {
                const int v = half + b;
                double *pb = s->phi + 2 * (size_t)b * d, *pv = s->phi + 2 * (size_t)v * d;
                chars_t bc, vc;
                lpn_chars(p, pb, full, -1, xh, sm, &bc, cfg->mbl_Nc, words);
                store_chars(p, cfg, lp, b, &bc);
                /* copy_trajectory_lpn + var_trajectory_lpn */
                memcpy(pv, pb, sizeof(double) * 2 * d);
                copy_stream(s, v, b);
                lp->eps_iters[v] = var_trajectory(p, cfg, lp, pb, pv, v, &bc, w, xh, sm, &lp->eps[v], words);
                /* calc_chars_lpn_start: delta_s from the std characteristics (calc_delta_f) */
                lpn_chars(p, pv, full, -1, xh, sm, &vc, cfg->mbl_Nc, words);
                store_chars(p, cfg, lp, v, &vc);
                lp->delta_s[v] = lpn_delta(p, cfg, &vc, &bc);
                lp->delta_s[b] = 0.0;
                lp->lambda[b] = lp->lambda[v] = 0.0;
                lp->lambda_now[b] = lp->lambda_now[v] = 0.0;
                lp->num_renorms[b] = lp->num_renorms[v] = 0;
                lp->renormed[b] = lp->renormed[v] = 0;
            }
        }
        free(w);
        free(xh);
        free(sm);
    }
    free(words);
    return bad;
}

/* LpnMultDeep sub-periods without a Lyapunov step: calc_chars_lpn of the bases only
 * (ex_period_obs_deep_mult_lpn, core.cpp:155-241). */
int orc_lpn_bases(const orc_problem *p, orc_state *s, const orc_lpn_config *cfg, orc_lpn *lp)
{
    const int d = p->d, n = p->n_traj, half = n / 2;
    if (!lpn_type_ok(p, cfg) || p->num_robs > 64 || (n & 1)) return 2;
    const int full = CH_MEAN | CH_ENERGY | CH_ROBS_ALL;
    int *words = lpn_words(cfg);
    if (cfg->mbl_Nc > 0 && !words) return 1;
    int bad = 0;
#pragma omp parallel
    {
        double *xh = (double *)malloc(sizeof(double) * 2 * d);
        double *sm = (double *)malloc(sizeof(double) * 2 * d);
        if (!xh || !sm) {
#pragma omp atomic write
            bad = 1;
        } else {
#pragma omp for schedule(dynamic, 1)
            for (int b = 0; b < half; b++) {
                chars_t bc;
                lpn_chars(p, s->phi + 2 * (size_t)b * d, full, -1, xh, sm, &bc, cfg->mbl_Nc, words);
                store_chars(p, cfg, lp, b, &bc);
            }
        }
        free(xh);
        free(sm);
    }
    free(words);
    return bad;
}

int orc_lpn_period(const orc_problem *p, orc_state *s, const orc_lpn_config *cfg, orc_lpn *lp, double curr_time)
{
    const int d = p->d, n = p->n_traj, half = n / 2;
    if (!lpn_type_ok(p, cfg) || p->num_robs > 64 || !s->rng_src || (n & 1)) return 2;
    const int full = CH_MEAN | CH_ENERGY | CH_ROBS_ALL;
    const int want = delta_want(cfg), one = delta_one(cfg);
    int *words = lpn_words(cfg);
    if (cfg->mbl_Nc > 0 && !words) return 1;
    int bad = 0;
#pragma omp parallel
    {
        double *w = (double *)malloc(sizeof(double) * 2 * d);
        double *xh = (double *)malloc(sizeof(double) * 2 * d);
        double *sm = (double *)malloc(sizeof(double) * 2 * d);
        if (!w || !xh || !sm) {
#pragma omp atomic write
            bad = 1;
        } else {
#pragma omp for schedule(dynamic, 1)
            for (int b = 0; b < half; b++) {
                const int v = half + b;
                double *pb = s->phi + 2 * (size_t)b * d, *pv = s->phi + 2 * (size_t)v * d;
                chars_t bc, vf, vc;
                /* calc_chars_lpn of the base (its std characteristics are the same numbers) */
                lpn_chars(p, pb, full, -1, xh, sm, &bc, cfg->mbl_Nc, words);
                store_chars(p, cfg, lp, b, &bc);
                /* calc_delta_f from the variation's std characteristics */
                lpn_chars(p, pv, want, one, xh, sm, &vf, cfg->mbl_Nc, words);
                const double df = lpn_delta(p, cfg, &vf, &bc);
                const double ds = lp->delta_s[v];
                const double ds10 = ds * 10.0;
                const double lim = (cfg->delta_f_high < ds10) ? ds10 : cfg->delta_f_high;  /* std::max */
                lp->renormed[v] = 0;
                if (cfg->per_period || df > lim || df < cfg->delta_f_low) {
                    const double ratio = df / ds;
                    lp->lambda[v] = lp->lambda[v] + orc_lpn_log(ratio + 1.0e-16);
                    lp->num_renorms[v] += 1;
                    lp->renormed[v] = 1;
                    lp->ratio[v] = ratio;
                    lp->ds_rec[v] = ds;
                    lp->df_rec[v] = df;
                    copy_stream(s, v, b);
                    lp->eps_iters[v] = var_trajectory(p, cfg, lp, pb, pv, v, &bc, w, xh, sm, &lp->eps[v], words);
                    lpn_chars(p, pv, full, -1, xh, sm, &vc, cfg->mbl_Nc, words);
                    store_chars(p, cfg, lp, v, &vc);
                    lp->delta_s[v] = lpn_delta(p, cfg, &vc, &bc);
                    lp->lambda_now[v] = lp->lambda[v] / curr_time;
                } else {
                    lpn_chars(p, pv, full, -1, xh, sm, &vc, cfg->mbl_Nc, words);
                    store_chars(p, cfg, lp, v, &vc);
                    lp->lambda_now[v] = (lp->lambda[v] + orc_lpn_log(df / ds + 1.0e-16)) / curr_time;
                }
            }
        }
        free(w);
        free(xh);
        free(sm);
    }
    free(words);
    return bad;
}
