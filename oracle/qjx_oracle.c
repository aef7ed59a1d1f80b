/*
 * qjx_oracle.c -- CPU restatement of the QJX QJ path (TEST INFRASTRUCTURE, see header).
 * Build: gcc -O3 -march=x86-64-v3 -ffp-contract=off -fopenmp -shared -fPIC (oracle/build_oracle.py).
 * -ffp-contract=off is part of the arithmetic contract: only the explicit fma() calls fuse.
 */
#include "qjx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ operators */

int orc_dimer_operators(int N, double J, double U, double E, double A, double g,
                        double *H, double *Hd, double *L, double *K0, double *K1)
{
    if (N < 1) return 1;
    const int d = N + 1;
    const size_t dd = (size_t)d * d;
    memset(H, 0, 2 * dd * sizeof(double));
    memset(Hd, 0, 2 * dd * sizeof(double));
    memset(L, 0, 2 * dd * sizeof(double));

    /* newdel.cpp:458-460: U is divided by (sys_size - 1) */
    const double Us = U / (double)(d - 1);
    for (int st = 0; st < d; st++) {
        size_t idx = (size_t)st * d + st;
        /* newdel.cpp:484-485 */
        H[2 * idx] = 2.0 * Us * (double)(st * (st - 1) + (d - (st + 1)) * (d - (st + 1) - 1));
        Hd[2 * idx] = (double)((d - (st + 1)) - st);
    }
    for (int st = 0; st < d - 1; st++) {
        size_t dl = (size_t)(st + 1) * d + st, ur = (size_t)st * d + (st + 1);
        /* newdel.cpp:493-494 */
        H[2 * dl] -= J * sqrt((double)((d - (st + 1)) * (st + 1)));
        H[2 * ur] -= J * sqrt((double)((st + 1) * (d - (st + 1))));
    }
    /* dissipator (newdel.cpp:1484-1497) */
    for (int st = 0; st < d; st++) {
        size_t idx = (size_t)st * d + st;
        L[2 * idx] = (double)(st - (d - (st + 1)));
    }
    for (int st = 0; st < d - 1; st++) {
        size_t dl = (size_t)(st + 1) * d + st, ur = (size_t)st * d + (st + 1);
        L[2 * dl] -= sqrt((double)((d - (st + 1)) * (st + 1)));
        L[2 * ur] += sqrt((double)((st + 1) * (d - (st + 1))));
    }

    /* newdel.cpp:2293-2294: gamma = g / (sys_size - 1) */
    const double gamma = g / (double)(d - 1);
    /* diss_part = gamma * L^H L (zgemm ConjTrans/NoTrans, newdel.cpp:2327-2342) */
    double *dp = (double *)malloc(2 * dd * sizeof(double));
    if (!dp) return 2;
    for (int i = 0; i < d; i++) {
        for (int j = 0; j < d; j++) {
            double sr = 0.0, si = 0.0;
            for (int k = 0; k < d; k++) {
                const double ar = L[2 * ((size_t)k * d + i)], ai = L[2 * ((size_t)k * d + i) + 1];
                const double br = L[2 * ((size_t)k * d + j)], bi = L[2 * ((size_t)k * d + j) + 1];
                sr = sr + (ar * br + ai * bi);
                si = si + (ar * bi - ai * br);
            }
            dp[2 * ((size_t)i * d + j)] = gamma * sr;
            dp[2 * ((size_t)i * d + j) + 1] = gamma * si;
        }
    }
    const double E0 = E + A, E1 = E - A; /* newdel.cpp:2369-2370 */
    for (size_t idx = 0; idx < dd; idx++) {
        /* hamitlonian_part = H - (i/2) diss_part  (newdel.cpp:2344-2352) */
        double hr = H[2 * idx] + 0.5 * dp[2 * idx + 1];
        double hi = 0.0 - 0.5 * dp[2 * idx];
        /* K_b = -i (hp + E_b Hd)  (newdel.cpp:2378-2382) */
        K0[2 * idx] = 0.0 + (hi + E0 * 0.0);
        K0[2 * idx + 1] = 0.0 - (hr + E0 * Hd[2 * idx]);
        K1[2 * idx] = 0.0 + (hi + E1 * 0.0);
        K1[2 * idx + 1] = 0.0 - (hr + E1 * Hd[2 * idx]);
    }
    free(dp);
    return 0;
}

/* JCS (sys_id 1): d = N; a = sum sqrt(k+1) |k><k+1| (newdel.cpp:608-614); H = 0.5 / alpha^3 ((a^+ a^+) a) a
 * (dgemm order, newdel.cpp:617-631); H_drv = a^+ - a; L = a (newdel.cpp:1571-1576); Nop = a^+ a
 * (experiment.cpp:2127-2135); gamma = 1 / (4 alpha), H_eff = H - (i/2) gamma L^H L,
 * K0 = -i H_eff + E0 H_drv, K1 = -i H_eff (newdel.cpp:2508-2597). */
static void rmatmul(int d, const double *A, const double *B, double *C)
{
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) {
            double s = 0.0;
            for (int k = 0; k < d; k++) s = s + A[(size_t)i * d + k] * B[(size_t)k * d + j];
            C[(size_t)i * d + j] = s;
        }
}

int orc_jcs_operators(int N, double alpha, double drv_ampl, double *H, double *Hd, double *L, double *Nop,
                      double *K0, double *K1)
{
    if (N < 2) return 1;
    const int d = N;
    const size_t dd = (size_t)d * d;
    double *a = (double *)calloc(dd, sizeof(double)), *ad = (double *)calloc(dd, sizeof(double));
    double *m1 = (double *)malloc(dd * sizeof(double)), *m2 = (double *)malloc(dd * sizeof(double));
    double *m3 = (double *)malloc(dd * sizeof(double)), *nop = (double *)malloc(dd * sizeof(double));
    if (!a || !ad || !m1 || !m2 || !m3 || !nop) return 2;
    for (int k = 0; k < d - 1; k++) {
        a[(size_t)k * d + (k + 1)] = sqrt((double)(k + 1));
        ad[(size_t)(k + 1) * d + k] = sqrt((double)(k + 1));
    }
    rmatmul(d, ad, ad, m1);
    rmatmul(d, m1, a, m2);
    rmatmul(d, m2, a, m3);
    rmatmul(d, ad, a, nop);
    const double hs = 0.5 / pow(alpha, 3);
    memset(H, 0, 2 * dd * sizeof(double));
    memset(Hd, 0, 2 * dd * sizeof(double));
    memset(L, 0, 2 * dd * sizeof(double));
    memset(Nop, 0, 2 * dd * sizeof(double));
    for (size_t e = 0; e < dd; e++) {
        H[2 * e] = hs * m3[e];
        Hd[2 * e] = ad[e] - a[e];
        L[2 * e] = a[e];
        Nop[2 * e] = nop[e];
    }
    const double gamma = 1.0 / (4.0 * alpha);
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) {
            double sr = 0.0, si = 0.0;
            for (int k = 0; k < d; k++) {
                const double ar = L[2 * ((size_t)k * d + i)], ai = L[2 * ((size_t)k * d + i) + 1];
                const double br = L[2 * ((size_t)k * d + j)], bi = L[2 * ((size_t)k * d + j) + 1];
                sr = sr + (ar * br + ai * bi);
                si = si + (ar * bi - ai * br);
            }
            const size_t idx = (size_t)i * d + j;
            const double hr = H[2 * idx] + 0.5 * (gamma * si);
            const double hi = 0.0 - 0.5 * (gamma * sr);
            K0[2 * idx] = 0.0 + (hi + drv_ampl * Hd[2 * idx]);
            K0[2 * idx + 1] = 0.0 - (hr + drv_ampl * 0.0);
            K1[2 * idx] = 0.0 + (hi + 0.0 * Hd[2 * idx]);
            K1[2 * idx + 1] = 0.0 - (hr + 0.0 * 0.0);
        }
    free(a); free(ad); free(m1); free(m2); free(m3); free(nop);
    return 0;
}

/* MBL (sys_id 3): Nc cells holding Nc/2 hard-core particles; the basis is every Nc-bit word with
 * Nc/2 bits set, in ascending order (MBLNewDelBehaviour::init_sizes, newdel.cpp:209-257). */
static int popcount_int(int v)
{
    int c = 0;
    while (v > 0) {
        c += v & 1;
        v >>= 1;
    }
    return c;
}

static int mbl_adjacent(int g) /* two set bits, neighbours (newdel.cpp:229-236) */
{
    return popcount_int(g) == 2 && popcount_int(g & (g << 1)) == 1;
}

int orc_mbl_basis(int Nc, int *id_to_x)
{
    if (Nc < 2 || Nc > 24 || Nc % 2) return -1;
    int n = 0;
    for (int x = 0; x < (1 << Nc); x++)
        if (popcount_int(x) == Nc / 2) {
            if (id_to_x) id_to_x[n] = x;
            n++;
        }
    return n;
}

/* MCG31m1 leapfrog stream (seed, k, s): u_i = x_{k+1+i s} / (2^31 - 1), x_n = 1132489760 x_{n-1}
 * mod 2^31 - 1 (the published MCG31m1 definition), mapped to [a, b) as a + (b - a) u. */
void orc_mcg31_uniform(unsigned long long seed, unsigned long long k, unsigned long long s, int count, double a,
                       double b, double *out)
{
    const unsigned long long m = 2147483647ull, mult = 1132489760ull;
    unsigned long long x = seed % m, p = 1, q = mult, e = k + 1, step = 1;
    if (x == 0) x = 1;
    while (e) { /* mult^(k+1) */
        if (e & 1) p = p * q % m;
        q = q * q % m;
        e >>= 1;
    }
    x = p * x % m;
    q = mult;
    e = s;
    while (e) { /* mult^s */
        if (e & 1) step = step * q % m;
        q = q * q % m;
        e >>= 1;
    }
    for (int i = 0; i < count; i++) {
        const double u = (double)x / (double)m;
        out[i] = a + (b - a) * u;
        x = x * step % m;
    }
}

/* MBL operators (newdel.cpp:868-958, 1699-1815, 2751-2838), d = C(Nc, Nc/2), basis words x_s:
 *   energies[c] : uniform(-1, 1) from MCG31 seed 77778888 leapfrogged (mbl_seed, mbl_mns)
 *   H  : diagonal W sum_c vb_c(x_s) energies[c] (vb_c = bit Nc-1-c), + U popcount(x & x << 1),
 *        then every element -= J [x_s ^ x_t holds two neighbouring bits]
 *   L_c: diss_type 0: diag(bit c of x_s), c < Nc; diss_type 1 (c < Nc-1): diag(bit c - bit c+1)
 *        plus the hop between the words that differ in bits c, c+1: -e^{-i phi} from the word
 *        with bit c set, e^{i phi} from the word with bit c+1 set
 *   K  : hamiltonians_qj[0] = -i (H - (i/2) sum_c gamma L_c^H L_c), jump rates g_c = 1.
 * L holds num_diss complex d x d matrices. */
int orc_mbl_operators(int Nc, double W, double U, double J, int mbl_seed, int mbl_mns, int diss_type, double diss_phase,
                      double gamma, double *energies, double *H, double *L, double *K)
{
    const int d = orc_mbl_basis(Nc, NULL);
    if (d < 2 || (diss_type != 0 && diss_type != 1)) return 1;
    const int nd = diss_type == 0 ? Nc : Nc - 1;
    const size_t dd = (size_t)d * d;
    int *xs = (int *)malloc((size_t)d * sizeof(int));
    double *hp = (double *)malloc(2 * dd * sizeof(double));
    if (!xs || !hp) return 2;
    orc_mbl_basis(Nc, xs);
    orc_mcg31_uniform(77778888ull, (unsigned long long)mbl_seed, (unsigned long long)mbl_mns, Nc, -1.0, 1.0, energies);
    memset(H, 0, 2 * dd * sizeof(double));
    memset(L, 0, 2 * dd * (size_t)nd * sizeof(double));
    for (int s = 0; s < d; s++) {
        double sum = 0.0;
        for (int c = 0; c < Nc; c++) sum += (double)((xs[s] >> (Nc - 1 - c)) & 1) * energies[c];
        sum *= 1.0 * W;
        H[2 * ((size_t)s * d + s)] += sum;
    }
    for (int s = 0; s < d; s++) H[2 * ((size_t)s * d + s)] += U * popcount_int(xs[s] & (xs[s] << 1));
    for (int s = 0; s < d; s++)
        for (int t = 0; t < d; t++) H[2 * ((size_t)s * d + t)] -= J * mbl_adjacent(xs[s] ^ xs[t]);
    for (int c = 0; c < nd; c++) {
        double *Lc = L + 2 * dd * (size_t)c;
        for (int s = 0; s < d; s++) {
            const int bc = (xs[s] >> c) & 1;
            Lc[2 * ((size_t)s * d + s)] = diss_type == 0 ? (double)bc : (double)bc - (double)((xs[s] >> (c + 1)) & 1);
        }
        if (diss_type == 0) continue;
        for (int s = 0; s < d; s++) {
            const int bc = (xs[s] >> c) & 1, bc1 = (xs[s] >> (c + 1)) & 1;
            if (bc == bc1) continue;
            for (int t = 0; t < d; t++) {
                const int g = xs[s] ^ xs[t];
                if (!mbl_adjacent(g) || (g & -g) != (1 << c)) continue; /* lower hop cell == c */
                double *e = Lc + 2 * ((size_t)s * d + t);
                if (bc) {
                    e[0] = -cos(-diss_phase);
                    e[1] = -sin(-diss_phase);
                } else {
                    e[0] = cos(diss_phase);
                    e[1] = sin(diss_phase);
                }
            }
        }
    }
    /* hamitlonian_part accumulates -(i/2) gamma L_c^H L_c channel by channel (newdel.cpp:2772-2828) */
    for (size_t e = 0; e < dd; e++) {
        hp[2 * e] = H[2 * e];
        hp[2 * e + 1] = 0.0;
    }
    for (int c = 0; c < nd; c++) {
        const double *Lc = L + 2 * dd * (size_t)c;
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                double sr = 0.0, si = 0.0;
                for (int k = 0; k < d; k++) {
                    const double ar = Lc[2 * ((size_t)k * d + i)], ai = Lc[2 * ((size_t)k * d + i) + 1];
                    const double br = Lc[2 * ((size_t)k * d + j)], bi = Lc[2 * ((size_t)k * d + j) + 1];
                    sr = sr + (ar * br + ai * bi);
                    si = si + (ar * bi - ai * br);
                }
                const size_t idx = (size_t)i * d + j;
                hp[2 * idx] += 0.5 * (gamma * si);
                hp[2 * idx + 1] -= 0.5 * (gamma * sr);
            }
    }
    for (size_t e = 0; e < dd; e++) {
        K[2 * e] = 0.0 + hp[2 * e + 1];
        K[2 * e + 1] = 0.0 - hp[2 * e];
    }
    free(xs);
    free(hp);
    return 0;
}

/* get_imbalance_mbl (experiment.cpp:1753-1800) for n trajectories' adr rows [n][d]:
 * n_c = sum_s adr_s vb_c(x_s) (s ascending), (sum_{c even} n_c - sum_{c odd} n_c) / total. */
void orc_mbl_imbalance(int Nc, int d, int n, const double *adr, double *out)
{
    int *xs = (int *)malloc((size_t)d * sizeof(int));
    double *np_ = (double *)malloc((size_t)Nc * sizeof(double));
    if (!xs || !np_) return;
    orc_mbl_basis(Nc, xs);
    for (int tr = 0; tr < n; tr++) {
        const double *a = adr + (size_t)tr * d;
        for (int c = 0; c < Nc; c++) np_[c] = 0.0;
        for (int s = 0; s < d; s++)
            for (int c = 0; c < Nc; c++) np_[c] += a[s] * (double)((xs[s] >> (Nc - 1 - c)) & 1);
        double so = 0.0, se = 0.0;
        for (int c = 0; c < Nc; c++) {
            if (c % 2 == 0) so += np_[c];
            else se += np_[c];
        }
        const double all = se + so;
        out[tr] = (so - se) / all;
    }
    free(xs);
    free(np_);
}

/* Integrable (sys_id 5, newdel.cpp:310-345, 1030-1095, 1924-2076, 2914-3004): N spins, d = 2^N, H = 0.
 * con = tau |00><00| + k |11><11| + |01><10| + |10><01| on neighbouring spins (c, c+1) for c < N-1
 * (kron order: spin 0 is the most significant bit), and on (N-1, 0) for the border channel;
 * special = y / sqrt(d), y = (X + X^H) / 2 normalised by sqrt(Re tr y^2), X_ij = g_ij (1 + i) with
 * g Box-Muller normals from MCG31 seed 13371337 leapfrogged (seed, num_seeds); K = -i (0 - (i/2)
 * sum_c L_c^H L_c), jump rates 1.  L holds N complex d x d matrices. */
int orc_integrable_operators(int N, int seed, int num_seeds, double tau, double kk, double *L, double *special,
                             double *K)
{
    if (N < 3 || N > 12) return 1;
    const int d = 1 << N;
    const size_t dd = (size_t)d * d;
    memset(L, 0, 2 * dd * (size_t)N * sizeof(double));
    /* channel c < N-1 acts on spins (c, c+1), i.e. bits (N-1-c, N-2-c); the border on (N-1, 0):
     * bits 0 (spin N-1, first of the pair) and N-1 (spin 0) */
    for (int c = 0; c < N; c++) {
        double *Lc = L + 2 * dd * (size_t)c;
        const int ba = c < N - 1 ? N - 1 - c : 0, bb = c < N - 1 ? N - 2 - c : N - 1;
        for (int s = 0; s < d; s++) {
            const int a = (s >> ba) & 1, b = (s >> bb) & 1;
            if (a == b) {
                Lc[2 * ((size_t)s * d + s)] = a ? kk : tau;
            } else {
                const int r = s ^ (1 << ba) ^ (1 << bb); /* |01> <-> |10> */
                Lc[2 * ((size_t)r * d + s)] = 1.0;
            }
        }
    }
    double *u = (double *)malloc(2 * dd * sizeof(double)), *g = (double *)malloc(dd * sizeof(double));
    double *y = (double *)malloc(2 * dd * sizeof(double)), *hp = (double *)malloc(2 * dd * sizeof(double));
    if (!u || !g || !y || !hp) return 2;
    orc_mcg31_uniform(13371337ull, (unsigned long long)seed, (unsigned long long)num_seeds, (int)(2 * dd), 0.0, 1.0, u);
    const double two_pi = 2.0 * 3.1415926535897932384626433832795;
    for (size_t e = 0; e < dd; e++) g[e] = sqrt(-2.0 * log(u[2 * e])) * sin(two_pi * u[2 * e + 1]);
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) { /* 0.5 (X + X^H), X_ij = g_ij + i g_ij */
            const double gij = g[(size_t)i * d + j], gji = g[(size_t)j * d + i];
            y[2 * ((size_t)i * d + j)] = 0.5 * (gij + gji);
            y[2 * ((size_t)i * d + j) + 1] = 0.5 * (gij + -gji);
        }
    double tr = 0.0; /* Re tr y^2: sum_i sum_k y_ik y_ki, k ascending, then i ascending */
    for (int i = 0; i < d; i++) {
        double sr = 0.0;
        for (int k = 0; k < d; k++) {
            const double ar = y[2 * ((size_t)i * d + k)], ai = y[2 * ((size_t)i * d + k) + 1];
            const double br = y[2 * ((size_t)k * d + i)], bi = y[2 * ((size_t)k * d + i) + 1];
            sr = sr + (ar * br - ai * bi);
        }
        tr = tr + sr;
    }
    const double sy = sqrt(tr), sd = sqrt((double)d);
    for (size_t e = 0; e < 2 * dd; e++) special[e] = (y[e] / sy) / sd;
    for (size_t e = 0; e < 2 * dd; e++) hp[e] = 0.0;
    for (int c = 0; c < N; c++) {
        const double *Lc = L + 2 * dd * (size_t)c;
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                double sr = 0.0, si = 0.0;
                for (int k = 0; k < d; k++) {
                    const double ar = Lc[2 * ((size_t)k * d + i)], ai = Lc[2 * ((size_t)k * d + i) + 1];
                    const double br = Lc[2 * ((size_t)k * d + j)], bi = Lc[2 * ((size_t)k * d + j) + 1];
                    sr = sr + (ar * br + ai * bi);
                    si = si + (ar * bi - ai * br);
                }
                const size_t idx = (size_t)i * d + j;
                hp[2 * idx] += 0.5 * (1.0 * si);
                hp[2 * idx + 1] -= 0.5 * (1.0 * sr);
            }
    }
    for (size_t e = 0; e < dd; e++) {
        K[2 * e] = 0.0 + hp[2 * e + 1];
        K[2 * e + 1] = 0.0 - hp[2 * e];
    }
    free(u);
    free(g);
    free(y);
    free(hp);
    return 0;
}

/* PS (sys_id 2, newdel.cpp:132-181, 650-866, 1582-1697, 2603-2749): ns spins (index x, spin 0 the most
 * significant bit) times nps photon states, basis index x nps + k (Kronecker order spins (x) photons).
 *   H  = (d/2) J_z (x) 1 + (g/2)(J_- (x) a^+ + J_+ (x) a) + 1 (x) (0.5/alpha^3) a^+a^+aa, J = sum sigma / 2
 *   Hd = 1 (x) (a^+ - a);  S = [1 (x) a, J_z (x) 1, J_+ (x) 1, 1 (x) a^+a] (spec, spec_2, spec_3, photons)
 *   L  = [1 (x) a] (+ [sigma_-^(s) (x) 1] for diss_type 1), H_eff with gamma 1/(4 alpha) for the
 *        cavity and diss_w for the spins; K0 = -i H_eff + E0 Hd (the kick), K1 = -i H_eff. */
int orc_ps_operators(int ns, int nps, double alpha, double dprm, double gprm, double drv_ampl, int diss_type,
                     double diss_w, double *H, double *Hd, double *L, double *S, double *K0, double *K1)
{
    if (ns < 1 || ns > 8 || nps < 2 || (diss_type != 0 && diss_type != 1)) return 1;
    const int n2 = 1 << ns, d = n2 * nps, nd = diss_type == 0 ? 1 : 1 + ns;
    const size_t dd = (size_t)d * d, pp = (size_t)nps * nps;
    double *a = (double *)calloc(pp, sizeof(double)), *ad = (double *)calloc(pp, sizeof(double));
    double *m1 = (double *)malloc(pp * sizeof(double)), *m2 = (double *)malloc(pp * sizeof(double));
    double *m3 = (double *)malloc(pp * sizeof(double)), *nop = (double *)malloc(pp * sizeof(double));
    double *jz = (double *)calloc((size_t)n2 * n2, sizeof(double)), *jm = (double *)calloc((size_t)n2 * n2, sizeof(double));
    double *jp = (double *)calloc((size_t)n2 * n2, sizeof(double)), *hp = (double *)malloc(2 * dd * sizeof(double));
    if (!a || !ad || !m1 || !m2 || !m3 || !nop || !jz || !jm || !jp || !hp) return 2;
    for (int k = 0; k < nps - 1; k++) {
        a[(size_t)k * nps + (k + 1)] = sqrt((double)(k + 1));
        ad[(size_t)(k + 1) * nps + k] = sqrt((double)(k + 1));
    }
    rmatmul(nps, ad, ad, m1);
    rmatmul(nps, m1, a, m2);
    rmatmul(nps, m2, a, m3);
    rmatmul(nps, ad, a, nop);
    const double hs = 0.5 / pow(alpha, 3);
    /* J_z, J_-, J_+: sums over spins of sigma_z = diag(1, -1), sigma_- = |1><0|, sigma_+ = |0><1| */
    for (int sp = 0; sp < ns; sp++)
        for (int x = 0; x < n2; x++) {
            const int bit = 1 << (ns - 1 - sp), b = (x & bit) != 0;
            jz[(size_t)x * n2 + x] += b ? -1.0 : 1.0;
            if (!b) jm[(size_t)(x | bit) * n2 + x] += 1.0;
            else jp[(size_t)(x & ~bit) * n2 + x] += 1.0;
        }
    for (size_t e = 0; e < (size_t)n2 * n2; e++) {
        jz[e] *= 0.5;
        jm[e] *= 0.5;
        jp[e] *= 0.5;
    }
    const double sd = dprm * 0.5, sg = gprm * 0.5;
    memset(H, 0, 2 * dd * sizeof(double));
    memset(Hd, 0, 2 * dd * sizeof(double));
    memset(L, 0, 2 * dd * (size_t)nd * sizeof(double));
    memset(S, 0, 8 * dd * sizeof(double));
    for (int xi = 0; xi < n2; xi++)
        for (int xj = 0; xj < n2; xj++)
            for (int ki = 0; ki < nps; ki++)
                for (int kj = 0; kj < nps; kj++) {
                    const size_t I = (size_t)xi * nps + ki, J = (size_t)xj * nps + kj, e = I * d + J;
                    const double id_s = xi == xj ? 1.0 : 0.0, id_p = ki == kj ? 1.0 : 0.0;
                    const size_t pe = (size_t)ki * nps + kj, se = (size_t)xi * n2 + xj;
                    const double s_ham = (sd * jz[se]) * id_p;
                    const double s_p = sg * (ad[pe] * jm[se] + jp[se] * a[pe]);
                    const double p_ham = id_s * (hs * m3[pe]);
                    H[2 * e] = (s_ham + s_p) + p_ham;
                    Hd[2 * e] = id_s * (ad[pe] - a[pe]);
                    S[2 * e] = id_s * a[pe];
                    S[2 * (dd + e)] = jz[se] * id_p;
                    S[2 * (2 * dd + e)] = jp[se] * id_p;
                    S[2 * (3 * dd + e)] = id_s * nop[pe];
                    L[2 * e] = id_s * a[pe];
                }
    if (diss_type == 1)
        for (int sp = 0; sp < ns; sp++) {
            double *Lc = L + 2 * dd * (size_t)(1 + sp);
            const int bit = 1 << (ns - 1 - sp);
            for (int x = 0; x < n2; x++)
                if (!(x & bit))
                    for (int k = 0; k < nps; k++)
                        Lc[2 * (((size_t)(x | bit) * nps + k) * d + (size_t)x * nps + k)] = 1.0;
        }
    for (size_t e = 0; e < dd; e++) {
        hp[2 * e] = H[2 * e];
        hp[2 * e + 1] = 0.0;
    }
    for (int c = 0; c < nd; c++) {
        const double *Lc = L + 2 * dd * (size_t)c;
        const double gamma = c == 0 ? 1.0 / (4.0 * alpha) : diss_w;
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                double sr = 0.0, si = 0.0;
                for (int k = 0; k < d; k++) {
                    const double ar = Lc[2 * ((size_t)k * d + i)], ai = Lc[2 * ((size_t)k * d + i) + 1];
                    const double br = Lc[2 * ((size_t)k * d + j)], bi = Lc[2 * ((size_t)k * d + j) + 1];
                    sr = sr + (ar * br + ai * bi);
                    si = si + (ar * bi - ai * br);
                }
                const size_t idx = (size_t)i * d + j;
                hp[2 * idx] += 0.5 * (gamma * si);
                hp[2 * idx + 1] -= 0.5 * (gamma * sr);
            }
    }
    for (size_t e = 0; e < dd; e++) {
        K0[2 * e] = 0.0 + (hp[2 * e + 1] + drv_ampl * Hd[2 * e]);
        K0[2 * e + 1] = 0.0 - (hp[2 * e] + drv_ampl * 0.0);
        K1[2 * e] = 0.0 + (hp[2 * e + 1] + 0.0 * Hd[2 * e]);
        K1[2 * e + 1] = 0.0 - (hp[2 * e] + 0.0 * 0.0);
    }
    free(a); free(ad); free(m1); free(m2); free(m3); free(nop); free(jz); free(jm); free(jp); free(hp);
    return 0;
}

/* Floq2Spins (sys_id 7, newdel.cpp:346-378, 1096-1182, 2077-2136, 3005-3101): two spins, d = 4 (spin 0
 * the more significant), H = (Delta_1 sz (x) 1 + Delta_2 1 (x) sz) / 2 + J sy (x) sy (real: diagonal
 * (Delta_1 s1 + Delta_2 s2) / 2, anti-diagonal -J, J, J, -J), special = H, L = [sm (x) 1, 1 (x) sm]
 * with sm = |1><0|, K = -i (H - (i/2) gamma sum L^H L); the drive enters the RK propagator only. */
int orc_floq2spins_operators(double D1, double D2, double J, double gamma, double *H, double *L, double *K)
{
    const int d = 4;
    const size_t dd = 16;
    memset(H, 0, 2 * dd * sizeof(double));
    memset(L, 0, 4 * dd * sizeof(double));
    for (int x = 0; x < d; x++) {
        const double s1 = (x & 2) ? -1.0 : 1.0, s2 = (x & 1) ? -1.0 : 1.0;
        H[2 * (x * d + x)] = 0.5 * (D1 * s1 + D2 * s2);
    }
    H[2 * (0 * d + 3)] = -J;
    H[2 * (1 * d + 2)] = J;
    H[2 * (2 * d + 1)] = J;
    H[2 * (3 * d + 0)] = -J;
    for (int x = 0; x < d; x++) {
        if (!(x & 2)) L[2 * ((x | 2) * d + x)] = 1.0;           /* sm on spin 0 */
        if (!(x & 1)) L[2 * (dd + (x | 1) * d + x)] = 1.0;      /* sm on spin 1 */
    }
    double hp[32];
    for (size_t e = 0; e < 2 * dd; e++) hp[e] = H[e];
    for (int c = 0; c < 2; c++) {
        const double *Lc = L + 2 * dd * c;
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                double sr = 0.0, si = 0.0;
                for (int k = 0; k < d; k++) {
                    const double ar = Lc[2 * (k * d + i)], ai = Lc[2 * (k * d + i) + 1];
                    const double br = Lc[2 * (k * d + j)], bi = Lc[2 * (k * d + j) + 1];
                    sr = sr + (ar * br + ai * bi);
                    si = si + (ar * bi - ai * br);
                }
                hp[2 * (i * d + j)] += 0.5 * (gamma * si);
                hp[2 * (i * d + j) + 1] -= 0.5 * (gamma * sr);
            }
    }
    for (size_t e = 0; e < dd; e++) {
        K[2 * e] = 0.0 + hp[2 * e + 1];
        K[2 * e + 1] = 0.0 - hp[2 * e];
    }
    return 0;
}

/* FloqManySpins (sys_id 8, newdel.cpp:379-413, 1184-1332, 2138-2224, 3103-3199): n spins, d = 2^n
 * (spin 0 the most significant bit); H = (Delta / 2) sum_s sz_s + J sy^(x)n for n >= 2, (Delta / 2)
 * sz for n = 1 (sy^(x)n couples x with x ^ (2^n - 1) by i^(n + 2 z(x)), z = zeros of x); special = H;
 * L_s = sm on spin s; K = -i (H - (i/2) gamma sum L^H L); the drive enters the RK propagator only. */
int orc_floqnspins_operators(int n, double Delta, double J, double gamma, double *H, double *L, double *K)
{
    if (n < 1 || n > 10) return 1;
    const int d = 1 << n;
    const size_t dd = (size_t)d * d;
    memset(H, 0, 2 * dd * sizeof(double));
    memset(L, 0, 2 * dd * (size_t)n * sizeof(double));
    const double hd = 0.5 * Delta;
    for (int x = 0; x < d; x++) {
        double sz = 0.0;
        int z = 0;
        for (int sp = 0; sp < n; sp++) {
            const int b = (x >> (n - 1 - sp)) & 1;
            sz = sz + (b ? -1.0 : 1.0);
            z += !b;
        }
        H[2 * ((size_t)x * d + x)] = (n == 1) ? hd * sz : sz * hd;
        if (n >= 2) {
            static const double ire[4] = {1.0, 0.0, -1.0, 0.0}, iim[4] = {0.0, 1.0, 0.0, -1.0};
            const int k = (n + 2 * z) & 3;
            const size_t e = (size_t)x * d + (x ^ (d - 1));
            H[2 * e] = J * ire[k];
            H[2 * e + 1] = J * iim[k];
        }
        for (int sp = 0; sp < n; sp++) {
            const int bit = 1 << (n - 1 - sp);
            if (!(x & bit)) L[2 * (dd * sp + (size_t)(x | bit) * d + x)] = 1.0;
        }
    }
    double *hp = (double *)malloc(2 * dd * sizeof(double));
    if (!hp) return 2;
    memcpy(hp, H, 2 * dd * sizeof(double));
    for (int c = 0; c < n; c++) {
        const double *Lc = L + 2 * dd * (size_t)c;
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                double sr = 0.0, si = 0.0;
                for (int k = 0; k < d; k++) {
                    const double ar = Lc[2 * ((size_t)k * d + i)], ai = Lc[2 * ((size_t)k * d + i) + 1];
                    const double br = Lc[2 * ((size_t)k * d + j)], bi = Lc[2 * ((size_t)k * d + j) + 1];
                    sr = sr + (ar * br + ai * bi);
                    si = si + (ar * bi - ai * br);
                }
                const size_t idx = (size_t)i * d + j;
                hp[2 * idx] += 0.5 * (gamma * si);
                hp[2 * idx + 1] -= 0.5 * (gamma * sr);
            }
    }
    for (size_t e = 0; e < dd; e++) {
        K[2 * e] = 0.0 + hp[2 * e + 1];
        K[2 * e + 1] = 0.0 - hp[2 * e];
    }
    free(hp);
    return 0;
}

/* FloqSpinPh (sys_id 9, newdel.cpp:414-449, 1334-1452, 2226-2284, 3201-3297): photons (x) spin, index
 * 2 k + s, d = 2 (n_ph + 1); H = (Delta / 2) 1 (x) sz + (Omega / 2)(a^+ (x) sm + a (x) sp), special = H,
 * L = a (x) 1, K = -i (H - (i/2) gamma L^H L); the drive enters the RK propagator only. */
int orc_floqspph_operators(int n_ph, double Delta, double Omega, double gamma, double *H, double *L, double *K)
{
    if (n_ph < 1) return 1;
    const int d = 2 * (n_ph + 1);
    const size_t dd = (size_t)d * d;
    memset(H, 0, 2 * dd * sizeof(double));
    memset(L, 0, 2 * dd * sizeof(double));
    const double hd = 0.5 * Delta, ho = 0.5 * Omega;
    for (int k = 0; k <= n_ph; k++) {
        H[2 * ((size_t)(2 * k) * d + 2 * k)] = hd * 1.0;
        H[2 * ((size_t)(2 * k + 1) * d + 2 * k + 1)] = hd * -1.0;
    }
    for (int k = 0; k < n_ph; k++) {
        const double a = sqrt((double)(k + 1));
        H[2 * ((size_t)(2 * (k + 1) + 1) * d + 2 * k)] = ho * a; /* a^+ (x) sm: (k, 0) -> (k + 1, 1) */
        H[2 * ((size_t)(2 * k) * d + 2 * (k + 1) + 1)] = ho * a; /* a (x) sp: (k + 1, 1) -> (k, 0) */
        for (int sp = 0; sp < 2; sp++) L[2 * ((size_t)(2 * k + sp) * d + 2 * (k + 1) + sp)] = a;
    }
    double *hp = (double *)malloc(2 * dd * sizeof(double));
    if (!hp) return 2;
    memcpy(hp, H, 2 * dd * sizeof(double));
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) {
            double sr = 0.0, si = 0.0;
            for (int k = 0; k < d; k++) {
                const double ar = L[2 * ((size_t)k * d + i)], ai = L[2 * ((size_t)k * d + i) + 1];
                const double br = L[2 * ((size_t)k * d + j)], bi = L[2 * ((size_t)k * d + j) + 1];
                sr = sr + (ar * br + ai * bi);
                si = si + (ar * bi - ai * br);
            }
            const size_t idx = (size_t)i * d + j;
            hp[2 * idx] += 0.5 * (gamma * si);
            hp[2 * idx + 1] -= 0.5 * (gamma * sr);
        }
    for (size_t e = 0; e < dd; e++) {
        K[2 * e] = 0.0 + hp[2 * e + 1];
        K[2 * e + 1] = 0.0 - hp[2 * e];
    }
    free(hp);
    return 0;
}

/* H_eff = H - (i/2) gamma L^H L (newdel.cpp:2327-2352), the RK propagator's non_drv_part */
int orc_dimer_heff(int N, double J, double U, double E, double g, double *Heff)
{
    const int d = N + 1;
    const size_t dd = (size_t)d * d;
    double *H = malloc(2 * dd * sizeof(double)), *Hd = malloc(2 * dd * sizeof(double));
    double *L = malloc(2 * dd * sizeof(double)), *K = malloc(4 * dd * sizeof(double));
    if (!H || !Hd || !L || !K) return 2;
    int rc = orc_dimer_operators(N, J, U, E, 0.0, g, H, Hd, L, K, K + 2 * dd);
    const double gamma = g / (double)(d - 1);
    for (int i = 0; i < d && !rc; i++)
        for (int j = 0; j < d; j++) {
            double sr = 0.0, si = 0.0;
            for (int k = 0; k < d; k++) {
                const double ar = L[2 * ((size_t)k * d + i)], ai = L[2 * ((size_t)k * d + i) + 1];
                const double br = L[2 * ((size_t)k * d + j)], bi = L[2 * ((size_t)k * d + j) + 1];
                sr = sr + (ar * br + ai * bi);
                si = si + (ar * bi - ai * br);
            }
            const size_t idx = (size_t)i * d + j;
            Heff[2 * idx] = H[2 * idx] + 0.5 * (gamma * si);
            Heff[2 * idx + 1] = 0.0 - 0.5 * (gamma * sr);
        }
    free(H); free(Hd); free(L); free(K);
    return rc;
}

/* ------------------------------------------------------------------ expm */

static void cmatmul(int n, const double *A, const double *B, double *C)
{
    /* C = A * B, complex row-major; i-k-j loop order */
    memset(C, 0, 2 * (size_t)n * n * sizeof(double));
    for (int i = 0; i < n; i++) {
        double *c = C + 2 * (size_t)i * n;
        for (int k = 0; k < n; k++) {
            const double ar = A[2 * ((size_t)i * n + k)], ai = A[2 * ((size_t)i * n + k) + 1];
            if (ar == 0.0 && ai == 0.0) continue;
            const double *b = B + 2 * (size_t)k * n;
            for (int j = 0; j < n; j++) {
                const double br = b[2 * j], bi = b[2 * j + 1];
                c[2 * j] += ar * br - ai * bi;
                c[2 * j + 1] += ar * bi + ai * br;
            }
        }
    }
}

/* out = sum_i c[i] * M_i + c0 * I   (M_i complex n x n, c real) */
static void lincomb(int n, int cnt, const double *c, const double *const *M, double c0, double *out)
{
    const size_t nn = (size_t)n * n;
    for (size_t e = 0; e < 2 * nn; e++) {
        double s = 0.0;
        for (int i = 0; i < cnt; i++) s += c[i] * M[i][e];
        out[e] = s;
    }
    for (int i = 0; i < n; i++) out[2 * ((size_t)i * n + i)] += c0;
}

/* Solve P X = Q (complex n x n) by Gaussian elimination with partial pivoting; Q is
 * overwritten with X, P is destroyed. */
static int csolve(int n, double *P, double *Q)
{
    for (int c = 0; c < n; c++) {
        int piv = c;
        double best = -1.0;
        for (int r = c; r < n; r++) {
            double v = hypot(P[2 * ((size_t)r * n + c)], P[2 * ((size_t)r * n + c) + 1]);
            if (v > best) { best = v; piv = r; }
        }
        if (best == 0.0) return 1;
        if (piv != c) {
            for (int j = 0; j < n; j++) {
                for (int q = 0; q < 2; q++) {
                    double t = P[2 * ((size_t)c * n + j) + q];
                    P[2 * ((size_t)c * n + j) + q] = P[2 * ((size_t)piv * n + j) + q];
                    P[2 * ((size_t)piv * n + j) + q] = t;
                    t = Q[2 * ((size_t)c * n + j) + q];
                    Q[2 * ((size_t)c * n + j) + q] = Q[2 * ((size_t)piv * n + j) + q];
                    Q[2 * ((size_t)piv * n + j) + q] = t;
                }
            }
        }
        const double pr = P[2 * ((size_t)c * n + c)], pi = P[2 * ((size_t)c * n + c) + 1];
        const double den = pr * pr + pi * pi;
        const double ir = pr / den, ii = -pi / den; /* 1 / pivot */
        for (int r = c + 1; r < n; r++) {
            const double ar = P[2 * ((size_t)r * n + c)], ai = P[2 * ((size_t)r * n + c) + 1];
            if (ar == 0.0 && ai == 0.0) continue;
            const double fr = ar * ir - ai * ii, fi = ar * ii + ai * ir;
            for (int j = c; j < n; j++) {
                const double br = P[2 * ((size_t)c * n + j)], bi = P[2 * ((size_t)c * n + j) + 1];
                P[2 * ((size_t)r * n + j)] -= fr * br - fi * bi;
                P[2 * ((size_t)r * n + j) + 1] -= fr * bi + fi * br;
            }
            for (int j = 0; j < n; j++) {
                const double br = Q[2 * ((size_t)c * n + j)], bi = Q[2 * ((size_t)c * n + j) + 1];
                Q[2 * ((size_t)r * n + j)] -= fr * br - fi * bi;
                Q[2 * ((size_t)r * n + j) + 1] -= fr * bi + fi * br;
            }
        }
    }
    for (int c = n - 1; c >= 0; c--) {
        const double pr = P[2 * ((size_t)c * n + c)], pi = P[2 * ((size_t)c * n + c) + 1];
        const double den = pr * pr + pi * pi;
        const double ir = pr / den, ii = -pi / den;
        for (int j = 0; j < n; j++) {
            double sr = Q[2 * ((size_t)c * n + j)], si = Q[2 * ((size_t)c * n + j) + 1];
            for (int k = c + 1; k < n; k++) {
                const double ar = P[2 * ((size_t)c * n + k)], ai = P[2 * ((size_t)c * n + k) + 1];
                const double xr = Q[2 * ((size_t)k * n + j)], xi = Q[2 * ((size_t)k * n + j) + 1];
                sr -= ar * xr - ai * xi;
                si -= ar * xi + ai * xr;
            }
            Q[2 * ((size_t)c * n + j)] = sr * ir - si * ii;
            Q[2 * ((size_t)c * n + j) + 1] = sr * ii + si * ir;
        }
    }
    return 0;
}

/* Pade coefficients b_0..b_m (Higham 2005, "The scaling and squaring method for the
 * matrix exponential revisited", SIAM J. Matrix Anal. Appl. 26(4)). */
static const double PADE3[] = {120.0, 60.0, 12.0, 1.0};
static const double PADE5[] = {30240.0, 15120.0, 3360.0, 420.0, 30.0, 1.0};
static const double PADE7[] = {17297280.0, 8648640.0, 1995840.0, 277200.0, 25200.0, 1512.0, 56.0, 1.0};
static const double PADE9[] = {17643225600.0, 8821612800.0, 2075673600.0, 302702400.0, 30270240.0,
                               2162160.0, 110880.0, 3960.0, 90.0, 1.0};
static const double PADE13[] = {64764752532480000.0, 32382376266240000.0, 7771770303897600.0,
                                1187353796428800.0, 129060195264000.0, 10559470521600.0,
                                670442572800.0, 33522128640.0, 1323241920.0, 40840800.0,
                                960960.0, 16380.0, 182.0, 1.0};
/* theta_m thresholds on ||A||_1 (Higham 2005, Table 2.3) */
static const double THETA[] = {1.495585217958292e-2, 2.539398330063230e-1, 9.504178996162932e-1,
                               2.097847961257068e0, 5.371920351148152e0};

int orc_expm(int n, const double *Ain, double *out)
{
    const size_t nn = (size_t)n * n, bytes = 2 * nn * sizeof(double);
    double *A = (double *)malloc(bytes), *A2 = (double *)malloc(bytes), *A4 = (double *)malloc(bytes);
    double *A6 = (double *)malloc(bytes), *W = (double *)malloc(bytes), *Uo = (double *)malloc(bytes);
    double *V = (double *)malloc(bytes), *T = (double *)malloc(bytes);
    if (!A || !A2 || !A4 || !A6 || !W || !Uo || !V || !T) return 2;
    memcpy(A, Ain, bytes);

    double l1 = 0.0;
    for (int j = 0; j < n; j++) {
        double s = 0.0;
        for (int i = 0; i < n; i++) s += hypot(A[2 * ((size_t)i * n + j)], A[2 * ((size_t)i * n + j) + 1]);
        if (s > l1) l1 = s;
    }
    int m, s = 0;
    if (l1 <= THETA[0]) m = 3;
    else if (l1 <= THETA[1]) m = 5;
    else if (l1 <= THETA[2]) m = 7;
    else if (l1 <= THETA[3]) m = 9;
    else {
        m = 13;
        s = (int)ceil(log2(l1 / THETA[4]));
        if (s < 0) s = 0;
        const double sc = ldexp(1.0, -s);
        for (size_t e = 0; e < 2 * nn; e++) A[e] *= sc;
    }

    cmatmul(n, A, A, A2);
    if (m == 3) {
        const double *M1[] = {A2};
        double c1[] = {PADE3[3]};
        lincomb(n, 1, c1, M1, PADE3[1], W);
        cmatmul(n, A, W, Uo);
        double c2[] = {PADE3[2]};
        lincomb(n, 1, c2, M1, PADE3[0], V);
    } else if (m == 5) {
        cmatmul(n, A2, A2, A4);
        const double *M1[] = {A4, A2};
        double cu[] = {PADE5[5], PADE5[3]}, cv[] = {PADE5[4], PADE5[2]};
        lincomb(n, 2, cu, M1, PADE5[1], W);
        cmatmul(n, A, W, Uo);
        lincomb(n, 2, cv, M1, PADE5[0], V);
    } else if (m == 7) {
        cmatmul(n, A2, A2, A4);
        cmatmul(n, A4, A2, A6);
        const double *M1[] = {A6, A4, A2};
        double cu[] = {PADE7[7], PADE7[5], PADE7[3]}, cv[] = {PADE7[6], PADE7[4], PADE7[2]};
        lincomb(n, 3, cu, M1, PADE7[1], W);
        cmatmul(n, A, W, Uo);
        lincomb(n, 3, cv, M1, PADE7[0], V);
    } else if (m == 9) {
        cmatmul(n, A2, A2, A4);
        cmatmul(n, A4, A2, A6);
        cmatmul(n, A6, A2, T); /* A8 */
        const double *M1[] = {T, A6, A4, A2};
        double cu[] = {PADE9[9], PADE9[7], PADE9[5], PADE9[3]};
        double cv[] = {PADE9[8], PADE9[6], PADE9[4], PADE9[2]};
        lincomb(n, 4, cu, M1, PADE9[1], W);
        cmatmul(n, A, W, Uo);
        lincomb(n, 4, cv, M1, PADE9[0], V);
    } else {
        cmatmul(n, A2, A2, A4);
        cmatmul(n, A4, A2, A6);
        const double *M3[] = {A6, A4, A2};
        /* U = A [A6 (b13 A6 + b11 A4 + b9 A2) + b7 A6 + b5 A4 + b3 A2 + b1 I] */
        double c_hi_u[] = {PADE13[13], PADE13[11], PADE13[9]};
        lincomb(n, 3, c_hi_u, M3, 0.0, T);
        cmatmul(n, A6, T, W);
        double c_lo_u[] = {PADE13[7], PADE13[5], PADE13[3]};
        lincomb(n, 3, c_lo_u, M3, PADE13[1], T);
        for (size_t e = 0; e < 2 * nn; e++) T[e] += W[e];
        cmatmul(n, A, T, Uo);
        /* V = A6 (b12 A6 + b10 A4 + b8 A2) + b6 A6 + b4 A4 + b2 A2 + b0 I */
        double c_hi_v[] = {PADE13[12], PADE13[10], PADE13[8]};
        lincomb(n, 3, c_hi_v, M3, 0.0, T);
        cmatmul(n, A6, T, W);
        double c_lo_v[] = {PADE13[6], PADE13[4], PADE13[2]};
        lincomb(n, 3, c_lo_v, M3, PADE13[0], V);
        for (size_t e = 0; e < 2 * nn; e++) V[e] += W[e];
    }
    /* (V - U) X = (V + U) */
    for (size_t e = 0; e < 2 * nn; e++) {
        const double u = Uo[e], v = V[e];
        T[e] = v - u;
        out[e] = v + u;
    }
    int rc = csolve(n, T, out);
    for (int k = 0; k < s && rc == 0; k++) {
        cmatmul(n, out, out, W);
        memcpy(out, W, bytes);
    }
    free(A); free(A2); free(A4); free(A6); free(W); free(Uo); free(V); free(T);
    return rc;
}

int orc_split_tree(int d, const double *K, double T, int deep, double *U_out)
{
    if (deep < 1) return 1;
    const size_t dd = (size_t)d * d;
    double *dts = (double *)malloc(sizeof(double) * deep);
    double dt = T * 0.5; /* qj_proc.cpp:15-16 */
    for (int l = 0; l < deep; l++) { dt *= 0.5; dts[l] = dt; }
    int rc = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : rc)
    for (int l = 0; l < deep; l++) {
        double *scaled = (double *)malloc(2 * dd * sizeof(double));
        for (size_t e = 0; e < dd; e++) {
            scaled[2 * e] = K[2 * e] * dts[l];
            scaled[2 * e + 1] = K[2 * e + 1] * dts[l];
        }
        rc |= orc_expm(d, scaled, U_out + 2 * dd * (size_t)l);
        free(scaled);
    }
    free(dts);
    return rc;
}

/* ------------------------------------------------------------------ Philox */

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

double orc_philox_uniform(uint64_t seed, uint64_t tr, uint64_t idx)
{
    const uint64_t blk = idx >> 1;
    const uint32_t ctr[4] = {(uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)tr, (uint32_t)(tr >> 32)};
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    orc_philox4x32_10(ctr, key, o);
    const uint32_t a = (idx & 1) ? o[2] : o[0];
    const uint32_t b = (idx & 1) ? o[3] : o[1];
    const uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
    return (double)(m + 1) * 0x1p-53;
}

/* ------------------------------------------------------------------ canonical kernels */

void orc_matvec(int d, const double *M, const double *x, double *out)
{
    for (int i = 0; i < d; i++) {
        const double *row = M + 2 * (size_t)i * d;
        double re = 0.0, im = 0.0;
        for (int k = 0; k < d; k++) {
            const double mr = row[2 * k], mi = row[2 * k + 1];
            const double xr = x[2 * k], xi = x[2 * k + 1];
            re = fma(mr, xr, re);
            re = fma(-mi, xi, re);
            im = fma(mr, xi, im);
            im = fma(mi, xr, im);
        }
        out[2 * i] = re;
        out[2 * i + 1] = im;
    }
}

/* Same arithmetic as orc_matvec on a transposed planar copy (MTr/MTi are [k][ld],
 * ld = d rounded up to ORC_RB); rows are processed ORC_RB at a time so the compiler
 * vectorises across rows.  Each output keeps its own k-ascending fma chain, so the
 * result is bit-identical to orc_matvec (fnmadd(a,b,c) == fma(-a,b,c) exactly). */
#define ORC_RB 8
#if defined(__AVX2__) && defined(__FMA__)
#include <immintrin.h>
static void matvec_t(int d, int ld, const double *MTr, const double *MTi, const double *x, double *out)
{
    for (int i0 = 0; i0 < d; i0 += ORC_RB) {
        __m256d re0 = _mm256_setzero_pd(), re1 = _mm256_setzero_pd();
        __m256d im0 = _mm256_setzero_pd(), im1 = _mm256_setzero_pd();
        for (int k = 0; k < d; k++) {
            const __m256d xr = _mm256_set1_pd(x[2 * k]), xi = _mm256_set1_pd(x[2 * k + 1]);
            const double *cr = MTr + (size_t)k * ld + i0, *ci = MTi + (size_t)k * ld + i0;
            const __m256d r0 = _mm256_loadu_pd(cr), r1 = _mm256_loadu_pd(cr + 4);
            const __m256d q0 = _mm256_loadu_pd(ci), q1 = _mm256_loadu_pd(ci + 4);
            re0 = _mm256_fmadd_pd(r0, xr, re0);  re1 = _mm256_fmadd_pd(r1, xr, re1);
            re0 = _mm256_fnmadd_pd(q0, xi, re0); re1 = _mm256_fnmadd_pd(q1, xi, re1);
            im0 = _mm256_fmadd_pd(r0, xi, im0);  im1 = _mm256_fmadd_pd(r1, xi, im1);
            im0 = _mm256_fmadd_pd(q0, xr, im0);  im1 = _mm256_fmadd_pd(q1, xr, im1);
        }
        double re[ORC_RB], im[ORC_RB];
        _mm256_storeu_pd(re, re0); _mm256_storeu_pd(re + 4, re1);
        _mm256_storeu_pd(im, im0); _mm256_storeu_pd(im + 4, im1);
        for (int r = 0; r < ORC_RB && i0 + r < d; r++) {
            out[2 * (i0 + r)] = re[r];
            out[2 * (i0 + r) + 1] = im[r];
        }
    }
}
#else
static void matvec_t(int d, int ld, const double *MTr, const double *MTi, const double *x, double *out)
{
    for (int i0 = 0; i0 < d; i0 += ORC_RB) {
        double re[ORC_RB] = {0}, im[ORC_RB] = {0};
        for (int k = 0; k < d; k++) {
            const double xr = x[2 * k], xi = x[2 * k + 1];
            const double *cr = MTr + (size_t)k * ld + i0, *ci = MTi + (size_t)k * ld + i0;
            for (int r = 0; r < ORC_RB; r++) {
                re[r] = fma(cr[r], xr, re[r]);
                re[r] = fma(-ci[r], xi, re[r]);
                im[r] = fma(cr[r], xi, im[r]);
                im[r] = fma(ci[r], xr, im[r]);
            }
        }
        for (int r = 0; r < ORC_RB && i0 + r < d; r++) {
            out[2 * (i0 + r)] = re[r];
            out[2 * (i0 + r) + 1] = im[r];
        }
    }
}
#endif

typedef struct { int ld; double *r, *i; } tmat;

static int tmat_make(int d, int count, const double *M, tmat *out)
{
    const int ld = (d + ORC_RB - 1) / ORC_RB * ORC_RB;
    const size_t per = (size_t)d * ld;
    out->ld = ld;
    out->r = (double *)calloc(per * (count > 0 ? count : 1), sizeof(double));
    out->i = (double *)calloc(per * (count > 0 ? count : 1), sizeof(double));
    if (!out->r || !out->i) return 1;
    for (int c = 0; c < count; c++)
        for (int i = 0; i < d; i++)
            for (int k = 0; k < d; k++) {
                const size_t src = (size_t)c * d * d + (size_t)i * d + k;
                out->r[per * c + (size_t)k * ld + i] = M[2 * src];
                out->i[per * c + (size_t)k * ld + i] = M[2 * src + 1];
            }
    return 0;
}

static void tmat_free(tmat *t) { free(t->r); free(t->i); }

/* Canonical 32-way reduction: lane l holds the literal running sum of the terms with index
 * l, l+32, l+64, ... (ascending); the 32 partial sums are then combined by an xor
 * butterfly, offsets 16, 8, 4, 2, 1 (q[l] = p[l] + p[l ^ off]).  Addition is commutative,
 * so every lane of a GPU warp ends with the value returned here. */
static double lanes_finish(double p[32])
{
    for (int off = 16; off >= 1; off >>= 1) {
        double q[32];
        for (int l = 0; l < 32; l++) q[l] = p[l] + p[l ^ off];
        memcpy(p, q, sizeof(q));
    }
    return p[0];
}

double orc_norm_square(int d, const double *x)
{
    double p[32] = {0};
    for (int i = 0; i < d; i++) {
        const double a = x[2 * i] * x[2 * i];
        const double b = x[2 * i + 1] * x[2 * i + 1];
        p[i & 31] = p[i & 31] + (a + b);
    }
    return lanes_finish(p);
}

/* Ensemble purity.  Order of operations: psi_hat = psi / sqrt(p) per element with the canonical
 * norm p; rho_ij accumulates trajectories in ascending order (re += a_r b_r, re += a_i b_i,
 * im += a_i b_r, im += -a_r b_i, each one fma) and is divided by n; purity = canonical squared
 * norm of rho flattened row-major.  calc_purity (CalcTraseRO2.cpp:57-75) computes Tr(rho rho)
 * of the f-basis density matrix; here rho is the trajectory average. */
double orc_purity(int d, int n, const double *psi, double *rho)
{
    double *acc = (double *)calloc((size_t)2 * d * d, sizeof(double));
    double *hat = (double *)malloc(sizeof(double) * 2 * (size_t)d);
    for (int tr = 0; tr < n; tr++) {
        const double *x = psi + (size_t)2 * d * tr;
        const double q = sqrt(orc_norm_square(d, x));
        for (int k = 0; k < 2 * d; k++) hat[k] = x[k] / q;
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                double *z = acc + 2 * ((size_t)i * d + j);
                const double ar = hat[2 * i], ai = hat[2 * i + 1], br = hat[2 * j], bi = hat[2 * j + 1];
                z[0] = fma(ar, br, z[0]);
                z[0] = fma(ai, bi, z[0]);
                z[1] = fma(ai, br, z[1]);
                z[1] = fma(-ar, bi, z[1]);
            }
    }
    for (size_t e = 0; e < (size_t)2 * d * d; e++) acc[e] = acc[e] / (double)n;
    const double pur = orc_norm_square(d * d, acc);
    if (rho) memcpy(rho, acc, sizeof(double) * 2 * (size_t)d * d);
    free(acc);
    free(hat);
    return pur;
}

/* ------------------------------------------------------------------ QJ engine */

typedef struct {
    const orc_problem *p;
    orc_state *s;
    int tr;
    int is_obs;
    double *phi, *aux, *res, *gn;
    const tmat *tU, *tL;
    const double *dt;   /* [num_branches][deep] split-level steps */
    int err;
} traj_ctx;

static double draw(traj_ctx *c)
{
    const orc_problem *p = c->p;
    int64_t *pos = &c->s->rng_pos[c->tr];
    /* the jump stream of trajectory tr, or the one it was copied from (vslCopyStream of the
     * Lyapunov tasks, experiment.cpp:2228-2246) */
    const int src = c->s->rng_src ? c->s->rng_src[c->tr] : c->tr;
    if (p->rng_kind == 0) return orc_philox_uniform(p->seed, p->tr_base + (uint64_t)src, (uint64_t)(*pos)++);
    const int64_t lo = p->inj_off[src], hi = p->inj_off[src + 1];
    if (lo + *pos >= hi) { c->err = 3; return 0.5; }
    return p->inj_u[lo + (*pos)++];
}

/* recovery (experiment.cpp:1273-1382) on aux */
static void recovery(traj_ctx *c)
{
    const orc_problem *p = c->p;
    const int d = p->d, k = p->num_diss;
    double *phi = c->aux;
    double norm = sqrt(orc_norm_square(d, phi));
    for (int st = 0; st < d; st++) {
        phi[2 * st] /= norm;
        phi[2 * st + 1] /= norm;
    }
    double tmp = 0.0, ran = draw(c);
    for (int i = 0; i < k; i++) {
        matvec_t(d, c->tL->ld, c->tL->r + (size_t)d * c->tL->ld * i, c->tL->i + (size_t)d * c->tL->ld * i, phi, c->res);
        c->s->matvecs[c->tr]++;
        c->gn[i] = orc_norm_square(d, c->res);
        c->gn[i] *= p->g[i];
        tmp += c->gn[i];
    }
    ran *= tmp;
    /* Same walk as experiment.cpp:1326-1334, with the index held below k - 1 before the
     * test (the reference's loop reads gnorms[1] when k == 1 and ran > gnorms[0], which
     * its own uniforms in [0,1) cannot produce; injected uniforms above 1 could). */
    int index = 0;
    while (index < k - 1 && ran - c->gn[index] > 0.0) {
        ran -= c->gn[index];
        index++;
    }
    if (tmp == 0.0) { c->err = 2; return; } /* reference would loop forever / read out of range */
    for (int it = 0; c->gn[index] == 0; it++) {
        if (it > 2 * k) { c->err = 2; return; }
        if (index == 0) index++;
        else index--;
        if (index >= k) { c->err = 2; return; }
    }
    matvec_t(d, c->tL->ld, c->tL->r + (size_t)d * c->tL->ld * index, c->tL->i + (size_t)d * c->tL->ld * index, phi, c->res);
    c->s->matvecs[c->tr]++;
    for (int st = 0; st < d; st++) {
        phi[2 * st] = c->res[2 * st] / sqrt(c->gn[index] / p->g[index]);
        phi[2 * st + 1] = c->res[2 * st + 1] / sqrt(c->gn[index] / p->g[index]);
    }
    if (p->record > 0 && c->is_obs == 1) {
        orc_state *s = c->s;
        int r = s->n_rec[c->tr] - 1; /* the record pushed just before this recovery */
        if (r >= 0 && r < s->rec_cap) s->diss_types[(size_t)c->tr * s->rec_cap + r] = index;
    }
}

/* one_period_branch (qj_proc.cpp:271-343), recursion over split levels */
static void one_period_branch(traj_ctx *c, int b, int level)
{
    const orc_problem *p = c->p;
    orc_state *s = c->s;
    const int d = p->d;
    const size_t dd = (size_t)d * d;
    const size_t moff = (size_t)d * c->tU->ld * ((size_t)b * p->deep + level);
    const double *Ur = c->tU->r + moff, *Ui = c->tU->i + moff;
    (void)dd;
    double *t = &s->t[c->tr];
    double *eta = &s->eta[c->tr];
    const double dt = c->dt[b * p->deep + level];

    if (level == p->deep - 1) {
        for (int counter = 0; counter != 2; counter++) {
            matvec_t(d, c->tU->ld, Ur, Ui, c->phi, c->aux);
            s->matvecs[c->tr]++;
            const double nrm = orc_norm_square(d, c->aux);
            if (nrm > 1.0) { c->err = 1; return; }
            if (!(nrm > *eta)) {
                if (p->record > 0 && c->is_obs == 1) {
                    const int r = s->n_rec[c->tr];
                    if (r >= s->rec_cap) { c->err = 4; return; }
                    const size_t o = (size_t)c->tr * s->rec_cap + r;
                    s->jump_times[o] = *t + dt;
                    s->jump_norms[o] = orc_norm_square(d, c->aux);
                    s->jump_etas[o] = *eta;
                    s->diss_types[o] = -1;
                    s->n_rec[c->tr] = r + 1;
                    s->jumps_counts[c->tr]++;
                }
                recovery(c);
                if (c->err) return;
                *eta = draw(c);
                while (*eta == 0.0) *eta = draw(c);
                if (c->err) return;
            }
            memcpy(c->phi, c->aux, 2 * (size_t)d * sizeof(double));
            *t += dt;
        }
    } else {
        for (int counter = 0; counter != 2; counter++) {
            matvec_t(d, c->tU->ld, Ur, Ui, c->phi, c->aux);
            s->matvecs[c->tr]++;
            const double nrm = orc_norm_square(d, c->aux);
            if (nrm > 1.0) { c->err = 1; return; }
            if (!(nrm > *eta)) {
                one_period_branch(c, b, level + 1);
                if (c->err) return;
                *t -= dt;
            } else {
                memcpy(c->phi, c->aux, 2 * (size_t)d * sizeof(double));
            }
            *t += dt;
        }
    }
}

int orc_init(const orc_problem *p, orc_state *s, int start_type, int start_state)
{
    const int d = p->d;
    for (int tr = 0; tr < p->n_traj; tr++) {
        double *phi = s->phi + 2 * (size_t)tr * d;
        memset(phi, 0, 2 * (size_t)d * sizeof(double));
        if (start_type == 0) phi[2 * start_state] = 1.0;
        else for (int i = 0; i < d; i++) phi[2 * i] = sqrt(1.0 / (double)d);
        s->t[tr] = 0.0;
        s->rng_pos[tr] = 0;
        s->jumps_counts[tr] = 0;
        s->matvecs[tr] = 0;
        s->n_rec[tr] = 0;
        s->error[tr] = 0;
        traj_ctx c = {0};
        c.p = p; c.s = s; c.tr = tr;
        s->eta[tr] = 0.0;
        while (s->eta[tr] == 0.0 && c.err == 0) s->eta[tr] = draw(&c);
        s->error[tr] = c.err;
    }
    return 0;
}

/* Split-level steps of every branch: level 0 steps half of the branch head H_b, every level
 * halves it (init_split_branches, qj_proc.cpp:15-24); H_b = 2 len_b, len_b = T / 2 by default. */
static double *dt_table(const orc_problem *p)
{
    double *t = (double *)malloc(sizeof(double) * (size_t)p->num_branches * p->deep);
    if (!t) return NULL;
    for (int b = 0; b < p->num_branches; b++) {
        double dt = (p->branch_len ? 2.0 * p->branch_len[b] : p->T) * 0.5;
        for (int l = 0; l < p->deep; l++) {
            dt *= 0.5;
            t[b * p->deep + l] = dt;
        }
    }
    return t;
}

int orc_run_periods(const orc_problem *p, orc_state *s, int tr0, int tr1, int n_periods, int is_obs, int n_threads)
{
    if (p->deep < 1 || p->deep > 60) return 1;
    int bad = 0;
    tmat tU, tL;
    if (tmat_make(p->d, p->num_branches * p->deep, p->U, &tU) || tmat_make(p->d, p->num_diss, p->L, &tL)) return 2;
    double *dtab = dt_table(p);
    if (!dtab) return 2;
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads) reduction(+ : bad)
#endif
    for (int tr = tr0; tr < tr1; tr++) {
        if (s->error[tr]) { bad++; continue; }
        const int d = p->d;
        traj_ctx c = {0};
        c.p = p; c.s = s; c.tr = tr; c.is_obs = is_obs;
        c.tU = &tU; c.tL = &tL;
        c.phi = s->phi + 2 * (size_t)tr * d;
        c.aux = (double *)calloc(2 * (size_t)d, sizeof(double));
        c.res = (double *)calloc(2 * (size_t)d, sizeof(double));
        c.gn = (double *)calloc((size_t)p->num_diss + 1, sizeof(double));
        c.dt = dtab;
        for (int per = 0; per < n_periods && !c.err; per++)
            for (int b = 0; b < p->num_branches && !c.err; b++) one_period_branch(&c, b, 0);
        s->error[tr] = c.err;
        if (c.err) bad++;
        free(c.aux); free(c.res); free(c.gn);
    }
    (void)n_threads;
    free(dtab);
    tmat_free(&tU);
    tmat_free(&tL);
    return bad;
}

/* n_units units of branch b (one_period_branch from level 0): the deep tasks' building block,
 * one sub-period being two units (one_sub_period_deep, qj_proc.cpp:345-359); p->T is the tree
 * head's dt, T / (2 deep_num_steps) for the deep tasks (core.cpp:9934). */
int orc_run_branch_units(const orc_problem *p, orc_state *s, int tr0, int tr1, int b, int n_units, int is_obs,
                         int n_threads)
{
    if (p->deep < 1 || p->deep > 60 || b < 0 || b >= p->num_branches) return 1;
    int bad = 0;
    tmat tU, tL;
    if (tmat_make(p->d, p->num_branches * p->deep, p->U, &tU) || tmat_make(p->d, p->num_diss, p->L, &tL)) return 2;
    double *dtab = dt_table(p);
    if (!dtab) return 2;
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads) reduction(+ : bad)
#endif
    for (int tr = tr0; tr < tr1; tr++) {
        if (s->error[tr]) { bad++; continue; }
        const int d = p->d;
        traj_ctx c = {0};
        c.p = p; c.s = s; c.tr = tr; c.is_obs = is_obs;
        c.tU = &tU; c.tL = &tL;
        c.phi = s->phi + 2 * (size_t)tr * d;
        c.aux = (double *)calloc(2 * (size_t)d, sizeof(double));
        c.res = (double *)calloc(2 * (size_t)d, sizeof(double));
        c.gn = (double *)calloc((size_t)p->num_diss + 1, sizeof(double));
        c.dt = dtab;
        for (int u = 0; u < n_units && !c.err; u++) one_period_branch(&c, b, 0);
        s->error[tr] = c.err;
        if (c.err) bad++;
        free(c.aux); free(c.res); free(c.gn);
    }
    (void)n_threads;
    free(dtab);
    tmat_free(&tU);
    tmat_free(&tL);
    return bad;
}

/* ------------------------------------------------------------------ RK propagator */

/* E(t) of rk_right_part_dimer (core.cpp:11073-11103) */
static double rk_drive(const orc_rk *rk, double T, double t)
{
    if (rk->drv_type == 1) return rk->E0 + rk->A * sin(rk->freq * t + rk->phase);
    const double mod_time = fmod(t, T), half_T = T * 0.5;
    return (mod_time < half_T) ? rk->E0 + rk->A : rk->E0 - rk->A;
}

typedef struct {
    traj_ctx *c;
    const orc_rk *rk;
    const tmat *tND, *tDR;
    double rk_step;
    double *prev, *args, *k1, *k2, *k3, *k4, *nd, *dr;
} rk_ctx;

/* k = -i (ND arg + E DR arg) (core.cpp:11106-11112) */
static void rk_right_part(rk_ctx *r, const double *arg, double t, double *k)
{
    traj_ctx *c = r->c;
    const int d = c->p->d;
    matvec_t(d, r->tND->ld, r->tND->r, r->tND->i, arg, r->nd);
    matvec_t(d, r->tDR->ld, r->tDR->r, r->tDR->i, arg, r->dr);
    c->s->matvecs[c->tr] += 2;
    const double E = rk_drive(r->rk, c->p->T, t);
    for (int st = 0; st < d; st++) {
        k[2 * st] = +(r->nd[2 * st + 1] + E * r->dr[2 * st + 1]);
        k[2 * st + 1] = -(r->nd[2 * st] + E * r->dr[2 * st]);
    }
}

/* rk_int_dimer (core.cpp:11592-11619) on c->phi with step h */
static void rk_int(rk_ctx *r, double h)
{
    traj_ctx *c = r->c;
    const int d = c->p->d;
    double *phi = c->phi, *t = &c->s->t[c->tr];
    const double rs = r->rk_step;
    memcpy(r->args, phi, 2 * (size_t)d * sizeof(double));
    rk_right_part(r, r->args, *t, r->k1);
    for (int e = 0; e < 2 * d; e++) r->args[e] = phi[e] + 0.5 * rs * r->k1[e];
    *t += h * 0.5;
    rk_right_part(r, r->args, *t, r->k2);
    for (int e = 0; e < 2 * d; e++) r->args[e] = phi[e] + 0.5 * rs * r->k2[e];
    rk_right_part(r, r->args, *t, r->k3);
    for (int e = 0; e < 2 * d; e++) r->args[e] = phi[e] + 1.0 * rs * r->k3[e];
    *t += h * 0.5;
    rk_right_part(r, r->args, *t, r->k4);
    for (int e = 0; e < 2 * d; e++) phi[e] += (r->k1[e] + 2.0 * r->k2[e] + 2.0 * r->k3[e] + r->k4[e]) * h / 6.0;
}

/* rk_step_dimer (core.cpp:11886-11948); its tail recursion on the end part is a loop here */
static void rk_step(rk_ctx *r, double h)
{
    traj_ctx *c = r->c;
    const orc_problem *p = c->p;
    orc_state *s = c->s;
    const int d = p->d;
    double *phi = c->phi, *t = &s->t[c->tr], *eta = &s->eta[c->tr];
    while (1) {
        memcpy(r->prev, phi, 2 * (size_t)d * sizeof(double));
        const double prev_norm = orc_norm_square(d, phi);
        rk_int(r, h);
        const double curr_norm = orc_norm_square(d, phi);
        if (curr_norm > 1.0) { c->err = 1; return; }
        if (curr_norm > *eta) return; /* not crossed */
        const double norm_diff = prev_norm - curr_norm;
        const double begin_part = (prev_norm - *eta) / norm_diff;
        const double end_part = 1.0 - begin_part;
        const double begin_step = h * begin_part, end_step = h * end_part;
        memcpy(phi, r->prev, 2 * (size_t)d * sizeof(double));
        *t -= h;
        rk_int(r, begin_step);
        if (p->record > 0 && c->is_obs == 1) {
            const int rr = s->n_rec[c->tr];
            if (rr >= s->rec_cap) { c->err = 4; return; }
            const size_t o = (size_t)c->tr * s->rec_cap + rr;
            s->jump_times[o] = *t;
            s->jump_norms[o] = orc_norm_square(d, phi);
            s->jump_etas[o] = *eta;
            s->diss_types[o] = -1;
            s->n_rec[c->tr] = rr + 1;
            s->jumps_counts[c->tr]++;
        }
        memcpy(c->aux, phi, 2 * (size_t)d * sizeof(double));
        recovery(c); /* rk_recovery (rk_proc.cpp:198-305): same steps as recovery */
        if (c->err) return;
        memcpy(phi, c->aux, 2 * (size_t)d * sizeof(double));
        *eta = draw(c);
        while (*eta == 0.0 && !c->err) *eta = draw(c);
        if (c->err) return;
        h = end_step;
    }
}

int orc_run_periods_rk(const orc_problem *p, const orc_rk *rk, orc_state *s, int tr0, int tr1, int n_periods,
                       int period0, int is_obs, int n_threads)
{
    if (rk->rk_ns < 1) return 1;
    int bad = 0;
    tmat tND, tDR, tL;
    if (tmat_make(p->d, 1, rk->ND, &tND) || tmat_make(p->d, 1, rk->DR, &tDR) || tmat_make(p->d, p->num_diss, p->L, &tL))
        return 2;
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads) reduction(+ : bad)
#endif
    for (int tr = tr0; tr < tr1; tr++) {
        if (s->error[tr]) { bad++; continue; }
        const int d = p->d;
        traj_ctx c = {0};
        c.p = p; c.s = s; c.tr = tr; c.is_obs = is_obs;
        c.tL = &tL;
        c.phi = s->phi + 2 * (size_t)tr * d;
        const size_t v = 2 * (size_t)d;
        double *buf = (double *)calloc(v * 11, sizeof(double));
        c.aux = buf;
        c.res = buf + v;
        c.gn = (double *)calloc((size_t)p->num_diss + 1, sizeof(double));
        rk_ctx r = {0};
        r.c = &c; r.rk = rk; r.tND = &tND; r.tDR = &tDR;
        r.rk_step = p->T / (double)rk->rk_ns;
        r.prev = buf + 2 * v; r.args = buf + 3 * v; r.k1 = buf + 4 * v; r.k2 = buf + 5 * v; r.k3 = buf + 6 * v;
        r.k4 = buf + 7 * v; r.nd = buf + 8 * v; r.dr = buf + 9 * v;
        for (int per = 0; per < n_periods && !c.err; per++)
            for (int sid = 0; sid < rk->rk_ns && !c.err; sid++) {
                s->t[tr] = (double)(period0 + per) * p->T + (double)sid * r.rk_step;
                rk_step(&r, r.rk_step);
            }
        s->error[tr] = c.err;
        if (c.err) bad++;
        free(buf); free(c.gn);
    }
    (void)n_threads;
    tmat_free(&tND);
    tmat_free(&tDR);
    tmat_free(&tL);
    return bad;
}

int orc_observables(const orc_problem *p, const orc_state *s, int is_start,
                    double *mean_start, double *norm_o, double *mean_o, double *disp_o,
                    double *m2_o, double *energy_o, double *robs, double *adr_o)
{
    const int d = p->d;
    tmat tH, tR;
    if (tmat_make(d, 1, p->HE, &tH) || tmat_make(d, p->num_robs, p->R, &tR)) return 2;
    const size_t per = (size_t)d * tH.ld;
#pragma omp parallel for schedule(static)
    for (int tr = 0; tr < p->n_traj; tr++) {
        const double *phi = s->phi + 2 * (size_t)tr * d;
        double *adr = (double *)malloc(sizeof(double) * d);
        double *xh = (double *)malloc(2 * sizeof(double) * d);
        double *sm = (double *)malloc(2 * sizeof(double) * d);
        const double norm = orc_norm_square(d, phi);
        for (int st = 0; st < d; st++) {
            /* mult_scalar_double(mult_scalar_complex(phi, phi, 1), 1/norm).real */
            const double a = phi[2 * st] * phi[2 * st], b = phi[2 * st + 1] * phi[2 * st + 1];
            adr[st] = (0.0 + (a + b)) * (1.0 / norm);
        }
        double ps[32] = {0};
        for (int st = 0; st < d; st++) ps[st & 31] = ps[st & 31] + (double)st * adr[st];
        const double mean = lanes_finish(ps);
        const double ms = is_start ? mean : mean_start[tr];
        const double disp = (mean - ms) * (mean - ms);
        memset(ps, 0, sizeof(ps));
        for (int st = 0; st < d; st++) ps[st & 31] = ps[st & 31] + ((double)st - mean) * ((double)st - mean) * adr[st];
        const double m2 = lanes_finish(ps);
        /* normalised state and energy <psi|H + E0 Hd|psi> (experiment.cpp:1423-1469) */
        const double sq = sqrt(norm);
        for (int st = 0; st < d; st++) {
            xh[2 * st] = phi[2 * st] / sq;
            xh[2 * st + 1] = phi[2 * st + 1] / sq;
        }
        matvec_t(d, tH.ld, tH.r, tH.i, xh, sm);
        memset(ps, 0, sizeof(ps));
        for (int st = 0; st < d; st++) {
            const double a = xh[2 * st] * sm[2 * st], b = xh[2 * st + 1] * sm[2 * st + 1];
            ps[st & 31] = ps[st & 31] + (a + b);
        }
        const double energy = lanes_finish(ps);
        /* random observables <psi|R|psi> (experiment.cpp:2023-2078) */
        for (int o = 0; o < p->num_robs; o++) {
            matvec_t(d, tR.ld, tR.r + per * o, tR.i + per * o, xh, sm);
            double pr[32] = {0}, pi[32] = {0};
            for (int st = 0; st < d; st++) {
                const double cr = xh[2 * st], ci = -xh[2 * st + 1];
                const double tr_ = cr * sm[2 * st] - ci * sm[2 * st + 1];
                const double ti_ = ci * sm[2 * st] + cr * sm[2 * st + 1];
                pr[st & 31] = pr[st & 31] + tr_;
                pi[st & 31] = pi[st & 31] + ti_;
            }
            const double rr = lanes_finish(pr), ri = lanes_finish(pi);
            robs[2 * ((size_t)tr * p->num_robs + o)] = rr;
            robs[2 * ((size_t)tr * p->num_robs + o) + 1] = ri;
        }
        if (is_start) mean_start[tr] = mean;
        norm_o[tr] = norm;
        mean_o[tr] = mean;
        disp_o[tr] = disp;
        m2_o[tr] = m2;
        energy_o[tr] = energy;
        if (adr_o) memcpy(adr_o + (size_t)tr * d, adr, sizeof(double) * d);
        free(adr); free(xh); free(sm);
    }
    tmat_free(&tH);
    tmat_free(&tR);
    return 0;
}

int orc_dump_periods(int dump_type, int dump_num, int num_obs_periods, int *periods)
{
    if (dump_type == 0) {
        periods[0] = 0;
        const int shift = num_obs_periods / dump_num;
        for (int i = 0; i < dump_num; i++) periods[i + 1] = (i + 1) * shift;
        return dump_num + 1;
    } else if (dump_type == 1) {
        periods[0] = 0;
        const double begin_decade = log10(1.0);
        const double end_decade = log10((double)num_obs_periods);
        const double num_decades = end_decade - begin_decade;
        const double num_decades_dump = (double)dump_num / num_decades;
        for (int i = 0; i < dump_num + 1; i++) {
            const int cur = (int)(pow(10.0, begin_decade) * pow(10.0, (1.0 / num_decades_dump) * (double)i));
            periods[i + 1] = cur > periods[i] ? cur : periods[i] + 1;
        }
        return dump_num + 2;
    }
    return -1;
}
