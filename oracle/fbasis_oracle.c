/*
 * fbasis_oracle.c -- CPU restatement of the SU(N) f-basis Lindblad solver of the dimer
 * (source/cpp/CQdiss_os_dimer), TEST INFRASTRUCTURE like qjx_oracle.c.
 *
 *   operators        create_H_base_matrix / create_H_drv_matrix (CQdiss/InitH.cpp:227-342),
 *                    init_diss L = A1 - i A2 (CQdiss/Init_a1_a2.cpp:6-122), gamma = g / N
 *                    (CQdiss/data.cpp:11)
 *   basis            index layout of initRhoODE / calcRho (CQdiss/calcODE.cpp:120-167,
 *                    CQdiss/CalcRho.cpp:4-67): for i < j the pair (sym, antisym), then the N
 *                    diagonal generalized Gell-Mann matrices; rho = I/d + sum_k x_k F_k
 *   Liouvillian      dx/dt = Gs x + E(t) Qs_drv x - Ks (CQdiss/calcODE.cpp:75-118).  The reference
 *                    assembles Gs = Qs_base + Rs and Ks from f/d structure constants
 *                    (CalcQs.cpp, CalcRs.cpp, CalcKs.cpp); here the same matrices are obtained by
 *                    projection, G_kl = Tr(F_k L0[F_l]) with L0 = -i[H_base, .] + D[.],
 *                    Qs_kl = Tr(F_k (-i[H_drv, F_l])), Ks_k = -Tr(F_k L0[I/d]).
 *   RK4              calcODE_trans / calcODE_std (CQdiss/calcODE.cpp:249-389), literal stage
 *                    arithmetic; the CSR row sum uses the canonical 32-lane order of the GPU
 *                    kernel (lane l sums nonzeros l, l+32, ... with fma, then an xor butterfly).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cplx;

/* f-basis flavour of the dimer operators (d = N + 1, complex row-major). */
int orc_fb_operators(int N, double J, double U, double E, double *Hb, double *Hdrv, double *L)
{
    const int d = N + 1;
    memset(Hb, 0, sizeof(double) * 2 * d * d);
    memset(Hdrv, 0, sizeof(double) * 2 * d * d);
    memset(L, 0, sizeof(double) * 2 * d * d);
    const double Ef = -E, Jf = -J; /* InitH.cpp:229-231 */
    double tr = 0.0;
    double *h2 = (double *)malloc(sizeof(double) * d);
    for (int i = 0; i < d; i++) {
        const double h1 = i * 2 - N;
        h2[i] = h1 * Ef + h1 * h1 * U / N;
        tr += h2[i];
    }
    tr /= (N + 1);
    for (int i = 0; i < d; i++) Hb[2 * (i * d + i)] = h2[i] - tr;
    for (int i = 1; i < d; i++) {
        Hb[2 * (i * d + i - 1)] = Jf * sqrt((double)((N - i + 1) * i));
        Hb[2 * ((i - 1) * d + i)] = Jf * sqrt((double)((N - i + 1) * i));
    }
    free(h2);
    for (int i = 0; i < d; i++) Hdrv[2 * (i * d + i)] = i * 2 - N; /* InitH.cpp:333-337 */
    /* L = A1 - i A2: A1 = diag(2i - N), A2(i,i-1) = -i sqrt((N-i+1) i), A2(i,i+1) = +i sqrt((N-i)(i+1)) */
    for (int i = 0; i < d; i++) L[2 * (i * d + i)] = 2.0 * i - N;
    for (int i = 0; i < N; i++) {
        const double s = sqrt((double)((N - i) * (i + 1)));
        L[2 * (i * d + i + 1)] = s;      /* -i * (+i s) */
        L[2 * ((i + 1) * d + i)] = -s;   /* -i * (-i s) */
    }
    return 0;
}

/* M (d x d complex) -> f coordinates Tr(F_k M) (real parts) */
static void project(int d, const cplx *M, double *out)
{
    const double v = 1.0 / sqrt(2.0);
    int k = 0;
    for (int i = 0; i < d; i++)
        for (int j = i + 1; j < d; j++) {
            out[k++] = (M[i * d + j].re + M[j * d + i].re) * v;
            /* Tr(F_anti M) = i (M_ji - M_ij) / sqrt 2 */
            out[k++] = -(M[j * d + i].im - M[i * d + j].im) * v;
        }
    for (int i = 0; i < d - 1; i++) {
        double s = 0.0;
        for (int j = 0; j <= i; j++) s += M[j * d + j].re;
        s -= (i + 1) * M[(i + 1) * d + (i + 1)].re;
        out[k++] = s / sqrt((double)((i + 1) * (i + 2)));
    }
}

/* basis element k as a dense matrix */
static void basis(int d, int k, cplx *F)
{
    memset(F, 0, sizeof(cplx) * d * d);
    const double v = 1.0 / sqrt(2.0);
    const int npairs = d * (d - 1) / 2;
    if (k < 2 * npairs) {
        int p = k / 2, i = 0;
        while (p >= d - 1 - i) { p -= d - 1 - i; i++; }
        const int j = i + 1 + p;
        if ((k & 1) == 0) { F[i * d + j].re = v; F[j * d + i].re = v; }
        else { F[i * d + j].im = v; F[j * d + i].im = -v; }
    } else {
        const int i = k - 2 * npairs;
        const double w = 1.0 / sqrt((double)((i + 1) * (i + 2)));
        for (int j = 0; j <= i; j++) F[j * d + j].re = w;
        F[(i + 1) * d + (i + 1)].re = -(i + 1) * w;
    }
}

static void cmul(int d, const cplx *A, const cplx *B, cplx *C)
{
    memset(C, 0, sizeof(cplx) * d * d);
    for (int i = 0; i < d; i++)
        for (int k = 0; k < d; k++) {
            const cplx a = A[i * d + k];
            if (a.re == 0.0 && a.im == 0.0) continue;
            for (int j = 0; j < d; j++) {
                const cplx b = B[k * d + j];
                C[i * d + j].re += a.re * b.re - a.im * b.im;
                C[i * d + j].im += a.re * b.im + a.im * b.re;
            }
        }
}

/* L0[X] = -i[Hb, X] + gamma (L X L^H - 1/2 {L^H L, X}); Ld = L^H, LdL = L^H L */
static void liou(int d, const cplx *Hb, const cplx *L, const cplx *Ld, const cplx *LdL, double gamma, const cplx *X,
                 cplx *out, cplx *t1, cplx *t2)
{
    cmul(d, Hb, X, t1);
    cmul(d, X, Hb, t2);
    for (int e = 0; e < d * d; e++) { /* -i (t1 - t2) */
        const double r = t1[e].re - t2[e].re, i = t1[e].im - t2[e].im;
        out[e].re = i;
        out[e].im = -r;
    }
    cmul(d, L, X, t1);
    cmul(d, t1, Ld, t2); /* L X L^H */
    for (int e = 0; e < d * d; e++) { out[e].re += gamma * t2[e].re; out[e].im += gamma * t2[e].im; }
    cmul(d, LdL, X, t1);
    cmul(d, X, LdL, t2);
    for (int e = 0; e < d * d; e++) {
        out[e].re -= 0.5 * gamma * (t1[e].re + t2[e].re);
        out[e].im -= 0.5 * gamma * (t1[e].im + t2[e].im);
    }
}

/* Dense f-basis matrices: Gs, Qs [n][n] row-major, Ks [n], n = d^2 - 1. */
int orc_fb_dense(int N, double J, double U, double E, double g, double *Gs, double *Qs, double *Ks)
{
    const int d = N + 1, n = d * d - 1;
    const double gamma = g / N;
    cplx *Hb = calloc(d * d, sizeof(cplx)), *Hd = calloc(d * d, sizeof(cplx)), *L = calloc(d * d, sizeof(cplx));
    cplx *Ld = calloc(d * d, sizeof(cplx)), *LdL = calloc(d * d, sizeof(cplx)), *Z = calloc(d * d, sizeof(cplx));
    cplx *F = calloc(d * d, sizeof(cplx)), *out = calloc(d * d, sizeof(cplx));
    cplx *t1 = calloc(d * d, sizeof(cplx)), *t2 = calloc(d * d, sizeof(cplx));
    double *col = malloc(sizeof(double) * n);
    if (!Hb || !Hd || !L || !Ld || !LdL || !Z || !F || !out || !t1 || !t2 || !col) return 2;
    orc_fb_operators(N, J, U, E, (double *)Hb, (double *)Hd, (double *)L);
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) { Ld[i * d + j].re = L[j * d + i].re; Ld[i * d + j].im = -L[j * d + i].im; }
    cmul(d, Ld, L, LdL);
    for (int l = 0; l < n; l++) {
        basis(d, l, F);
        liou(d, Hb, L, Ld, LdL, gamma, F, out, t1, t2);
        project(d, out, col);
        for (int k = 0; k < n; k++) Gs[(size_t)k * n + l] = col[k];
        liou(d, Hd, L, Ld, LdL, 0.0, F, out, t1, t2); /* -i[Hdrv, F] */
        project(d, out, col);
        for (int k = 0; k < n; k++) Qs[(size_t)k * n + l] = col[k];
    }
    memset(F, 0, sizeof(cplx) * d * d);
    for (int i = 0; i < d; i++) F[i * d + i].re = 1.0 / d;
    liou(d, Hb, L, Ld, LdL, gamma, F, out, t1, t2);
    project(d, out, col);
    for (int k = 0; k < n; k++) Ks[k] = -col[k];
    free(Hb); free(Hd); free(L); free(Ld); free(LdL); free(Z); free(F); free(out); free(t1); free(t2); free(col);
    return 0;
}

/* canonical CSR row product (shared with the GPU kernel) */
static double row_dot(const int *rp, const int *ci, const double *v, const double *x, int row)
{
    double p[32];
    for (int l = 0; l < 32; l++) p[l] = 0.0;
    const int b = rp[row], e = rp[row + 1];
    for (int j = b; j < e; j++) {
        const int l = (j - b) & 31;
        p[l] = fma(v[j], x[ci[j]], p[l]);
    }
    for (int off = 16; off >= 1; off >>= 1) {
        double q[32];
        for (int l = 0; l < 32; l++) q[l] = p[l] + p[l ^ off];
        memcpy(p, q, sizeof(q));
    }
    return p[0];
}

/* calcVectValue_real (calcODE.cpp:75-118) */
static void vect_value(int n, const int *gr, const int *gc, const double *gv, const int *qr, const int *qc,
                       const double *qv, const double *Ks, double drv_ampl, double freq, double phase, int drv_type,
                       double t, double h, const double *x, double *res)
{
    for (int i = 0; i < n; i++) {
        const double t1 = row_dot(gr, gc, gv, x, i), t2 = row_dot(qr, qc, qv, x, i);
        if (drv_type == 1) res[i] = (t1 + drv_ampl * sin(freq * t + phase) * t2 - Ks[i]) * h;
        else if (sin(freq * t + phase) < 0.0) res[i] = (t1 + drv_ampl * (-1.0) * t2 - Ks[i]) * h;
        else res[i] = (t1 + drv_ampl * (+1.0) * t2 - Ks[i]) * h;
    }
}

/* n_periods periods of num_steps RK4 steps from period0 (calcODE.cpp:270-303); drv_ampl is A
 * (the reference uses -A, calcODE.cpp:91). */
int orc_fb_rk4(int n, const int *gr, const int *gc, const double *gv, const int *qr, const int *qc, const double *qv,
               const double *Ks, double A, double freq, double phase, int drv_type, double T, int num_steps,
               int period0, int n_periods, double *x)
{
    double *k1 = malloc(sizeof(double) * n), *k2 = malloc(sizeof(double) * n), *k3 = malloc(sizeof(double) * n);
    double *k4 = malloc(sizeof(double) * n), *val = malloc(sizeof(double) * n);
    if (!k1 || !k2 || !k3 || !k4 || !val) return 2;
    const double step = T / (double)num_steps, amp = -A;
    for (int period = period0; period < period0 + n_periods; period++)
        for (int s = 0; s < num_steps; s++) {
            const double time = period * T + s * step;
            vect_value(n, gr, gc, gv, qr, qc, qv, Ks, amp, freq, phase, drv_type, time, step, x, k1);
            for (int i = 0; i < n; i++) val[i] = x[i] + k1[i] / 2.0;
            vect_value(n, gr, gc, gv, qr, qc, qv, Ks, amp, freq, phase, drv_type, time + step / 2.0, step, val, k2);
            for (int i = 0; i < n; i++) val[i] = x[i] + k2[i] / 2.0;
            vect_value(n, gr, gc, gv, qr, qc, qv, Ks, amp, freq, phase, drv_type, time + step / 2.0, step, val, k3);
            for (int i = 0; i < n; i++) val[i] = x[i] + k3[i];
            vect_value(n, gr, gc, gv, qr, qc, qv, Ks, amp, freq, phase, drv_type, time + step, step, val, k4);
            for (int i = 0; i < n; i++) x[i] += (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]) / 6.0;
        }
    free(k1); free(k2); free(k3); free(k4); free(val);
    return 0;
}

/* calcRho (CalcRho.cpp:4-67): rho = I/d + sum x_k F_k, complex row-major */
void orc_fb_rho(int N, const double *x, double *rho)
{
    const int d = N + 1;
    memset(rho, 0, sizeof(double) * 2 * d * d);
    for (int i = 0; i < d; i++) rho[2 * (i * d + i)] = 1.0 / d;
    int k = 0;
    double v = 1.0 / sqrt(2.0);
    for (int i = 0; i < d; i++)
        for (int j = i + 1; j < d; j++) {
            rho[2 * (i * d + j)] += x[k] * v;
            rho[2 * (j * d + i)] += x[k] * v;
            k++;
            rho[2 * (i * d + j) + 1] += x[k] * v;
            rho[2 * (j * d + i) + 1] += x[k] * (-v);
            k++;
        }
    for (int i = 0; i < N; i++) {
        v = 1.0 / sqrt((double)((i + 1) * (i + 2)));
        int j;
        for (j = 0; j <= i; j++) rho[2 * (j * d + j)] += x[k] * v;
        rho[2 * (j * d + j)] -= x[k] * v * (i + 1);
        k++;
    }
}

/* initRhoODE (calcODE.cpp:120-167), literally (its antisymmetric entries use the opposite
 * sign to calcRho; the start states of the reference are real and diagonal). */
void orc_fb_x_from_rho(int N, const double *rho, double *x)
{
    const int d = N + 1, n = d * d - 1;
    memset(x, 0, sizeof(double) * n);
    int k = 0;
    double v = 1.0 / sqrt(2.0);
    for (int i = 0; i < d; i++)
        for (int j = i + 1; j < d; j++) {
            x[k] += rho[2 * (i * d + j)] * v;
            x[k] += rho[2 * (j * d + i)] * v;
            k++;
            x[k] += rho[2 * (i * d + j) + 1] * (-v);
            x[k] += rho[2 * (j * d + i) + 1] * (+v);
            k++;
        }
    for (int i = 0; i < N; i++) {
        v = 1.0 / sqrt((double)((i + 1) * (i + 2)));
        for (int j = 0; j <= i; j++) x[k] += rho[2 * (j * d + j)] * v;
        x[k] -= rho[2 * ((i + 1) * d + (i + 1))] * v * (i + 1);
        k++;
    }
}
