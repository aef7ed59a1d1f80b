// qjx_model.cpp -- host construction of the dimer model and its split propagators (FP64).
//
// DimerNewDelBehaviour (source/cpp/QJX/QJX/newdel.cpp):
//   init_sizes            :3-37     d = N + 1, T = 2 pi / omega, one jump operator, two branches
//   init_hamiltonians     :450-498  H (interaction 2 (U/N) [k(k-1) + (N-k)(N-k-1)], hopping -J sqrt),
//                                    H_drv = diag(N - 2k)
//   init_dissipators      :1454-1498 L = diag(2k - N) + sqrt((k+1)(N-k)) (|k><k+1| - |k+1><k|)
//   init_hamiltonians_qj  :2285-2388 K_b = -i (H - i/2 gamma L^H L + E_b H_drv), gamma = g/N,
//                                    E_0 = E + A (first half period), E_1 = E - A
// init_split_branches (source/cpp/QJX/QJX/qj_proc.cpp:4-120): U_{b,l} = exp(K_b dt_l),
// dt_l = T 2^-(l+2).  The reference uses Eigen's MatrixXcd::exp(); this file implements the
// same published method (Higham 2005 scaling and squaring with diagonal Pade approximants).
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/qjx_b200.h"
#include "qjx_config.h"

namespace {

using cvec = std::vector<double>;  // interleaved complex, row-major

void matmul(int n, const double *A, const double *B, double *C)
{
    std::memset(C, 0, sizeof(double) * 2 * (size_t)n * n);
    for (int i = 0; i < n; i++) {
        double *c = C + 2 * (size_t)i * n;
        for (int k = 0; k < n; k++) {
            const double ar = A[2 * ((size_t)i * n + k)], ai = A[2 * ((size_t)i * n + k) + 1];
            if (ar == 0.0 && ai == 0.0) continue;
            const double *b = B + 2 * (size_t)k * n;
            for (int j = 0; j < n; j++) {
                c[2 * j] += ar * b[2 * j] - ai * b[2 * j + 1];
                c[2 * j + 1] += ar * b[2 * j + 1] + ai * b[2 * j];
            }
        }
    }
}

// out = sum_i c_i M_i + c0 I
void combine(int n, const std::vector<const double *> &M, const std::vector<double> &c, double c0, double *out)
{
    const size_t e2 = 2 * (size_t)n * n;
    for (size_t e = 0; e < e2; e++) {
        double s = 0.0;
        for (size_t i = 0; i < M.size(); i++) s += c[i] * M[i][e];
        out[e] = s;
    }
    for (int i = 0; i < n; i++) out[2 * ((size_t)i * n + i)] += c0;
}

// Solves P X = Q by LU with partial pivoting (P destroyed, X returned in Q).
bool solve(int n, double *P, double *Q)
{
    auto at = [n](double *M, int r, int c) { return M + 2 * ((size_t)r * n + c); };
    for (int c = 0; c < n; c++) {
        int piv = c;
        double best = -1.0;
        for (int r = c; r < n; r++) {
            const double v = std::hypot(at(P, r, c)[0], at(P, r, c)[1]);
            if (v > best) {
                best = v;
                piv = r;
            }
        }
        if (best == 0.0) return false;
        if (piv != c)
            for (int j = 0; j < n; j++)
                for (int q = 0; q < 2; q++) {
                    std::swap(at(P, c, j)[q], at(P, piv, j)[q]);
                    std::swap(at(Q, c, j)[q], at(Q, piv, j)[q]);
                }
        const double pr = at(P, c, c)[0], pi = at(P, c, c)[1], den = pr * pr + pi * pi;
        const double ir = pr / den, ii = -pi / den;
        for (int r = c + 1; r < n; r++) {
            const double ar = at(P, r, c)[0], ai = at(P, r, c)[1];
            if (ar == 0.0 && ai == 0.0) continue;
            const double fr = ar * ir - ai * ii, fi = ar * ii + ai * ir;
            for (int j = c; j < n; j++) {
                const double br = at(P, c, j)[0], bi = at(P, c, j)[1];
                at(P, r, j)[0] -= fr * br - fi * bi;
                at(P, r, j)[1] -= fr * bi + fi * br;
            }
            for (int j = 0; j < n; j++) {
                const double br = at(Q, c, j)[0], bi = at(Q, c, j)[1];
                at(Q, r, j)[0] -= fr * br - fi * bi;
                at(Q, r, j)[1] -= fr * bi + fi * br;
            }
        }
    }
    for (int c = n - 1; c >= 0; c--) {
        const double pr = at(P, c, c)[0], pi = at(P, c, c)[1], den = pr * pr + pi * pi;
        const double ir = pr / den, ii = -pi / den;
        for (int j = 0; j < n; j++) {
            double sr = at(Q, c, j)[0], si = at(Q, c, j)[1];
            for (int k = c + 1; k < n; k++) {
                const double ar = at(P, c, k)[0], ai = at(P, c, k)[1];
                const double xr = at(Q, k, j)[0], xi = at(Q, k, j)[1];
                sr -= ar * xr - ai * xi;
                si -= ar * xi + ai * xr;
            }
            at(Q, c, j)[0] = sr * ir - si * ii;
            at(Q, c, j)[1] = sr * ii + si * ir;
        }
    }
    return true;
}

// Diagonal Pade coefficients b_0..b_m and thresholds theta_m on ||A||_1 from Higham (2005).
const double kB3[] = {120.0, 60.0, 12.0, 1.0};
const double kB5[] = {30240.0, 15120.0, 3360.0, 420.0, 30.0, 1.0};
const double kB7[] = {17297280.0, 8648640.0, 1995840.0, 277200.0, 25200.0, 1512.0, 56.0, 1.0};
const double kB9[] = {17643225600.0, 8821612800.0, 2075673600.0, 302702400.0, 30270240.0,
                      2162160.0,     110880.0,     3960.0,       90.0,        1.0};
const double kB13[] = {64764752532480000.0, 32382376266240000.0, 7771770303897600.0, 1187353796428800.0,
                       129060195264000.0,   10559470521600.0,    670442572800.0,     33522128640.0,
                       1323241920.0,        40840800.0,          960960.0,           16380.0,
                       182.0,               1.0};
const double kTheta[] = {1.495585217958292e-2, 2.539398330063230e-1, 9.504178996162932e-1, 2.097847961257068e0,
                         5.371920351148152e0};

bool expm(int n, const double *Ain, double *out)
{
    const size_t e2 = 2 * (size_t)n * n;
    cvec A(Ain, Ain + e2), A2(e2), A4(e2), A6(e2), A8(e2), W(e2), T(e2), Uo(e2), V(e2);
    double l1 = 0.0;
    for (int j = 0; j < n; j++) {
        double s = 0.0;
        for (int i = 0; i < n; i++) s += std::hypot(A[2 * ((size_t)i * n + j)], A[2 * ((size_t)i * n + j) + 1]);
        l1 = std::max(l1, s);
    }
    int m = 13, sq = 0;
    if (l1 <= kTheta[0]) m = 3;
    else if (l1 <= kTheta[1]) m = 5;
    else if (l1 <= kTheta[2]) m = 7;
    else if (l1 <= kTheta[3]) m = 9;
    else {
        sq = std::max(0, (int)std::ceil(std::log2(l1 / kTheta[4])));
        const double sc = std::ldexp(1.0, -sq);
        for (double &x : A) x *= sc;
    }
    matmul(n, A.data(), A.data(), A2.data());
    if (m == 3) {
        combine(n, {A2.data()}, {kB3[3]}, kB3[1], W.data());
        matmul(n, A.data(), W.data(), Uo.data());
        combine(n, {A2.data()}, {kB3[2]}, kB3[0], V.data());
    } else if (m == 5) {
        matmul(n, A2.data(), A2.data(), A4.data());
        combine(n, {A4.data(), A2.data()}, {kB5[5], kB5[3]}, kB5[1], W.data());
        matmul(n, A.data(), W.data(), Uo.data());
        combine(n, {A4.data(), A2.data()}, {kB5[4], kB5[2]}, kB5[0], V.data());
    } else if (m == 7) {
        matmul(n, A2.data(), A2.data(), A4.data());
        matmul(n, A4.data(), A2.data(), A6.data());
        combine(n, {A6.data(), A4.data(), A2.data()}, {kB7[7], kB7[5], kB7[3]}, kB7[1], W.data());
        matmul(n, A.data(), W.data(), Uo.data());
        combine(n, {A6.data(), A4.data(), A2.data()}, {kB7[6], kB7[4], kB7[2]}, kB7[0], V.data());
    } else if (m == 9) {
        matmul(n, A2.data(), A2.data(), A4.data());
        matmul(n, A4.data(), A2.data(), A6.data());
        matmul(n, A6.data(), A2.data(), A8.data());
        combine(n, {A8.data(), A6.data(), A4.data(), A2.data()}, {kB9[9], kB9[7], kB9[5], kB9[3]}, kB9[1],
                W.data());
        matmul(n, A.data(), W.data(), Uo.data());
        combine(n, {A8.data(), A6.data(), A4.data(), A2.data()}, {kB9[8], kB9[6], kB9[4], kB9[2]}, kB9[0],
                V.data());
    } else {
        matmul(n, A2.data(), A2.data(), A4.data());
        matmul(n, A4.data(), A2.data(), A6.data());
        const std::vector<const double *> M3 = {A6.data(), A4.data(), A2.data()};
        combine(n, M3, {kB13[13], kB13[11], kB13[9]}, 0.0, T.data());
        matmul(n, A6.data(), T.data(), W.data());
        combine(n, M3, {kB13[7], kB13[5], kB13[3]}, kB13[1], T.data());
        for (size_t e = 0; e < e2; e++) T[e] += W[e];
        matmul(n, A.data(), T.data(), Uo.data());
        combine(n, M3, {kB13[12], kB13[10], kB13[8]}, 0.0, T.data());
        matmul(n, A6.data(), T.data(), W.data());
        combine(n, M3, {kB13[6], kB13[4], kB13[2]}, kB13[0], V.data());
        for (size_t e = 0; e < e2; e++) V[e] += W[e];
    }
    for (size_t e = 0; e < e2; e++) {
        T[e] = V[e] - Uo[e];
        out[e] = V[e] + Uo[e];
    }
    if (!solve(n, T.data(), out)) return false;
    for (int k = 0; k < sq; k++) {
        matmul(n, out, out, W.data());
        std::memcpy(out, W.data(), sizeof(double) * e2);
    }
    return true;
}

}  // namespace

extern "C" qjx_status qjx_expm(int n, const double *A, double *out)
{
    if (n < 1 || !A || !out) return QJX_ERR_INVALID_ARG;
    return expm(n, A, out) ? QJX_OK : QJX_ERR_INVALID_ARG;
}

// H_eff = H - (i/2) gamma L^H L (newdel.cpp:2327-2352) of real L; returns (hr, hi) of element (i, j)
static void heff_element(int d, const cvec &h, const cvec &l, double gamma, int i, int j, double &hr, double &hi)
{
    double sr = 0.0, si = 0.0;
    for (int k = 0; k < d; k++) {
        const double ar = l[2 * ((size_t)k * d + i)], ai = l[2 * ((size_t)k * d + i) + 1];
        const double br = l[2 * ((size_t)k * d + j)], bi = l[2 * ((size_t)k * d + j) + 1];
        sr = sr + (ar * br + ai * bi);
        si = si + (ar * bi - ai * br);
    }
    const size_t idx = (size_t)i * d + j;
    hr = h[2 * idx] + 0.5 * (gamma * si);
    hi = 0.0 - 0.5 * (gamma * sr);
}

static qjx_status build_dimer_impl(int N, double J, double U, double E, double A, double g, double omega, int deep,
                                   int deep_num_steps, double *H, double *Hd, double *L, double *Kout, double *Utree);

extern "C" qjx_status qjx_build_dimer(int N, double J, double U, double E, double A, double g, double omega,
                                      int deep, double *H, double *Hd, double *L, double *Kout, double *Utree)
{
    return build_dimer_impl(N, J, U, E, A, g, omega, deep, 0, H, Hd, L, Kout, Utree);
}

// Deep tasks: the split tree of a sub-period T_sub = T / (2 deep_num_steps)
// (init_split_structure_dimer_deep, core.cpp:9928-9940).
extern "C" qjx_status qjx_build_dimer_deep(int N, double J, double U, double E, double A, double g, double omega,
                                           int deep, int deep_num_steps, double *H, double *Hd, double *L,
                                           double *Kout, double *Utree)
{
    if (deep_num_steps < 1) return QJX_ERR_INVALID_ARG;
    return build_dimer_impl(N, J, U, E, A, g, omega, deep, deep_num_steps, H, Hd, L, Kout, Utree);
}

static qjx_status build_dimer_impl(int N, double J, double U, double E, double A, double g, double omega, int deep,
                                   int deep_num_steps, double *H, double *Hd, double *L, double *Kout, double *Utree)
{
    if (N < 1 || deep < 1 || !(omega > 0.0)) return QJX_ERR_INVALID_ARG;
    const int d = N + 1;
    const size_t dd = (size_t)d * d, e2 = 2 * dd;
    cvec h(e2, 0.0), hd(e2, 0.0), l(e2, 0.0);
    const double Us = U / double(d - 1);
    for (int k = 0; k < d; k++) {
        const size_t ii = 2 * ((size_t)k * d + k);
        h[ii] = 2.0 * Us * double(k * (k - 1) + (d - (k + 1)) * (d - (k + 1) - 1));
        hd[ii] = double((d - (k + 1)) - k);
        l[ii] = double(k - (d - (k + 1)));
    }
    for (int k = 0; k < d - 1; k++) {
        const size_t dl = 2 * ((size_t)(k + 1) * d + k), ur = 2 * ((size_t)k * d + (k + 1));
        const double s = std::sqrt(double((d - (k + 1)) * (k + 1)));
        h[dl] -= J * s;
        h[ur] -= J * s;
        l[dl] -= s;
        l[ur] += s;
    }
    if (H) std::memcpy(H, h.data(), e2 * sizeof(double));
    if (Hd) std::memcpy(Hd, hd.data(), e2 * sizeof(double));
    if (L) std::memcpy(L, l.data(), e2 * sizeof(double));
    if (!Utree && !Kout) return QJX_OK;

    // gamma L^H L (real L), H_eff = H - i/2 gamma L^H L, K_b = -i (H_eff + E_b H_drv)
    const double gamma = g / double(d - 1);
    cvec K[2] = {cvec(e2), cvec(e2)};
    const double Eb[2] = {E + A, E - A};
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) {
            const size_t idx = (size_t)i * d + j;
            double hr, hi;
            heff_element(d, h, l, gamma, i, j, hr, hi);
            for (int b = 0; b < 2; b++) {
                K[b][2 * idx] = 0.0 + (hi + Eb[b] * 0.0);
                K[b][2 * idx + 1] = 0.0 - (hr + Eb[b] * hd[2 * idx]);
            }
        }
    if (Kout) {
        std::memcpy(Kout, K[0].data(), e2 * sizeof(double));
        std::memcpy(Kout + e2, K[1].data(), e2 * sizeof(double));
    }
    if (!Utree) return QJX_OK;
    const double Tp = 2.0 * 3.1415926535897932384626433832795 / omega;
    const double T = deep_num_steps > 0 ? 0.5 * Tp / double(deep_num_steps) : Tp;  // the tree head's dt
    std::vector<double> dts(deep);
    double dt = T * 0.5;
    for (int lv = 0; lv < deep; lv++) {
        dt *= 0.5;
        dts[lv] = dt;
    }
    bool ok = true;
#pragma omp parallel for schedule(dynamic, 1) collapse(2) reduction(&& : ok)
    for (int b = 0; b < 2; b++)
        for (int lv = 0; lv < deep; lv++) {
            cvec scaled(e2);
            for (size_t e = 0; e < dd; e++) {
                scaled[2 * e] = K[b][2 * e] * dts[lv];
                scaled[2 * e + 1] = K[b][2 * e + 1] * dts[lv];
            }
            ok = expm(d, scaled.data(), Utree + e2 * ((size_t)b * deep + lv)) && ok;
        }
    return ok ? QJX_OK : QJX_ERR_INVALID_ARG;
}

// Operators of the RK propagator: H_eff = non_drv_part and H_drv = drv_part (newdel.cpp:2354-2366).
extern "C" qjx_status qjx_build_dimer_rk(int N, double J, double U, double E, double g, double *H_eff, double *H_drv)
{
    if (N < 1 || !H_eff || !H_drv) return QJX_ERR_INVALID_ARG;
    const int d = N + 1;
    const size_t e2 = 2 * (size_t)d * d;
    cvec h(e2), hd(e2), l(e2);
    const qjx_status st = qjx_build_dimer(N, J, U, E, 0.0, g, 1.0, 1, h.data(), hd.data(), l.data(), nullptr, nullptr);
    if (st != QJX_OK) return st;
    const double gamma = g / double(d - 1);
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) {
            const size_t idx = (size_t)i * d + j;
            heff_element(d, h, l, gamma, i, j, H_eff[2 * idx], H_eff[2 * idx + 1]);
        }
    std::memcpy(H_drv, hd.data(), e2 * sizeof(double));
    return QJX_OK;
}

// JCS (sys_id 1): JCSNewDelBehaviour (source/cpp/QJX/QJX/newdel.cpp)
//   init_sizes            :96-130   d = N, T = jcs_prm_alpha, one jump operator, two branches
//   init_hamiltonians     :564-649  H = 0.5 / alpha^3 a^+ a^+ a a, H_drv = a^+ - a, special = a
//   init_dissipators      :1546-1580 L = a
//   init_hamiltonians_qj  :2499-2601 gamma = 1 / (4 alpha); H_eff = H - i/2 gamma L^H L;
//                                     K_0 = -i H_eff + E0 H_drv (kick), K_1 = -i H_eff
// init_split_structure_jcs (core.cpp:10086-10124): branch b's head is jcs_drv_part_b * T, so
// U_{b,l} = exp(K_b head_b 2^-(l+2)) and branch b lasts head_b / 2.
// Products of the ladder matrices follow the reference's dgemm order ((a^+ a^+) a) a; each entry
// has a single nonzero term, so the order of the zero terms does not matter.
static void real_matmul(int d, const std::vector<double> &A, const std::vector<double> &B, std::vector<double> &C)
{
    C.assign((size_t)d * d, 0.0);
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) {
            double s = 0.0;
            for (int k = 0; k < d; k++) s = s + A[(size_t)i * d + k] * B[(size_t)k * d + j];
            C[(size_t)i * d + j] = s;
        }
}

extern "C" qjx_status qjx_build_jcs(int N, double alpha, double drv_ampl, double part_1, double part_2, int deep,
                                    double *H, double *Hd, double *L, double *Nop, double *A_op, double *Kout,
                                    double *Utree)
{
    if (N < 2 || !(alpha > 0.0) || deep < 1 || !(part_1 > 0.0) || !(part_2 > 0.0)) return QJX_ERR_INVALID_ARG;
    const int d = N;
    const size_t dd = (size_t)d * d, e2 = 2 * dd;
    std::vector<double> a(dd, 0.0), ad(dd, 0.0), m1, m2, m3, nop;
    for (int k = 0; k < d - 1; k++) {
        a[(size_t)k * d + (k + 1)] = std::sqrt(double(k + 1));
        ad[(size_t)(k + 1) * d + k] = std::sqrt(double(k + 1));
    }
    real_matmul(d, ad, ad, m1);
    real_matmul(d, m1, a, m2);
    real_matmul(d, m2, a, m3);
    real_matmul(d, ad, a, nop);  // get_num_photons_jcs (experiment.cpp:2080-2160)
    cvec h(e2, 0.0), hd(e2, 0.0), l(e2, 0.0);
    const double hs = 0.5 / std::pow(alpha, 3);
    for (size_t e = 0; e < dd; e++) {
        h[2 * e] = hs * m3[e];
        hd[2 * e] = ad[e] - a[e];
        l[2 * e] = a[e];
    }
    if (H) std::memcpy(H, h.data(), e2 * sizeof(double));
    if (Hd) std::memcpy(Hd, hd.data(), e2 * sizeof(double));
    if (L) std::memcpy(L, l.data(), e2 * sizeof(double));
    if (Nop)
        for (size_t e = 0; e < dd; e++) {
            Nop[2 * e] = nop[e];
            Nop[2 * e + 1] = 0.0;
        }
    if (A_op) std::memcpy(A_op, l.data(), e2 * sizeof(double));
    if (!Utree && !Kout) return QJX_OK;
    const double gamma = 1.0 / (4.0 * alpha);
    cvec K[2] = {cvec(e2), cvec(e2)};
    const double Eb[2] = {drv_ampl, 0.0};
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) {
            const size_t idx = (size_t)i * d + j;
            double hr, hi;
            heff_element(d, h, l, gamma, i, j, hr, hi);
            for (int b = 0; b < 2; b++) {
                K[b][2 * idx] = 0.0 + (hi + Eb[b] * hd[2 * idx]);
                K[b][2 * idx + 1] = 0.0 - (hr + Eb[b] * 0.0);
            }
        }
    if (Kout) {
        std::memcpy(Kout, K[0].data(), e2 * sizeof(double));
        std::memcpy(Kout + e2, K[1].data(), e2 * sizeof(double));
    }
    if (!Utree) return QJX_OK;
    const double head[2] = {part_1 * alpha, part_2 * alpha};
    bool ok = true;
#pragma omp parallel for schedule(dynamic, 1) collapse(2) reduction(&& : ok)
    for (int b = 0; b < 2; b++)
        for (int lv = 0; lv < deep; lv++) {
            double dt = head[b] * 0.5;
            for (int q = 0; q <= lv; q++) dt *= 0.5;
            cvec scaled(e2);
            for (size_t e = 0; e < dd; e++) {
                scaled[2 * e] = K[b][2 * e] * dt;
                scaled[2 * e + 1] = K[b][2 * e + 1] * dt;
            }
            ok = expm(d, scaled.data(), Utree + e2 * ((size_t)b * deep + lv)) && ok;
        }
    return ok ? QJX_OK : QJX_ERR_INVALID_ARG;
}

// ---------------------------------------------------------------------------------------- MBL
// MBLNewDelBehaviour (source/cpp/QJX/QJX/newdel.cpp): Nc cells, Nc/2 hard-core particles; the
// basis is every Nc-bit word with Nc/2 bits set, ascending (init_sizes :209-257).

static int bits_set(int v)
{
    int c = 0;
    for (; v > 0; v >>= 1) c += v & 1;
    return c;
}

// Two set bits that are neighbours: the words x, y are one hop apart iff x ^ y is such a pair.
static bool one_hop(int g) { return bits_set(g) == 2 && bits_set(g & (g << 1)) == 1; }

static std::vector<int> mbl_words(int Nc)
{
    std::vector<int> xs;
    for (int x = 0; x < (1 << Nc); x++)
        if (bits_set(x) == Nc / 2) xs.push_back(x);
    return xs;
}

extern "C" qjx_status qjx_mbl_size(int Nc, int diss_type, int *d, int *num_diss)
{
    if (Nc < 2 || Nc > 24 || Nc % 2 || (diss_type != 0 && diss_type != 1)) return QJX_ERR_INVALID_ARG;
    // C(Nc, Nc/2) by the multiplicative formula, exact in integers at every step
    long long c = 1;
    for (int i = 0; i < Nc / 2; i++) c = c * (Nc - i) / (i + 1);
    if (d) *d = int(c);
    if (num_diss) *num_diss = diss_type == 0 ? Nc : Nc - 1;
    return QJX_OK;
}

extern "C" qjx_status qjx_build_mbl(int Nc, double W, double U, double J, int mbl_seed, int mbl_mns, int diss_type,
                                    double diss_phase, double gamma, double T, int deep, double *energies,
                                    int *id_to_x, double *H, double *L, double *Kout, double *Utree)
{
    int d = 0, nd = 0;
    if (qjx_mbl_size(Nc, diss_type, &d, &nd) != QJX_OK || mbl_mns < 1 || mbl_seed < 0) return QJX_ERR_INVALID_ARG;
    if (Utree && (deep < 1 || !(T > 0.0))) return QJX_ERR_INVALID_ARG;
    const std::vector<int> xs = mbl_words(Nc);
    const size_t dd = (size_t)d * d, e2 = 2 * dd;
    // disorder (init_hamiltonians :891-905): uniform(-1, 1) from MCG31 seed 77778888, leapfrog
    // stream (mbl_seed, mbl_mns), as a + (b - a) u
    std::vector<double> en(Nc);
    qjxio::LeapfrogLCG st = qjxio::LeapfrogLCG::mcg31(77778888ull, (unsigned long long)mbl_seed,
                                                        (unsigned long long)mbl_mns);
    for (int c = 0; c < Nc; c++) en[c] = -1.0 + (1.0 - -1.0) * st.next();
    cvec h(e2, 0.0), l(e2 * nd, 0.0);
    for (int s = 0; s < d; s++) {  // W sum_c n_c e_c, cell c = bit Nc-1-c (:907-918)
        double sum = 0.0;
        for (int c = 0; c < Nc; c++) sum += double((xs[s] >> (Nc - 1 - c)) & 1) * en[c];
        sum *= 1.0 * W;
        h[2 * ((size_t)s * d + s)] += sum;
    }
    for (int s = 0; s < d; s++)  // U n_c n_{c+1} (:924-928)
        h[2 * ((size_t)s * d + s)] += U * bits_set(xs[s] & (xs[s] << 1));
    for (int s = 0; s < d; s++)  // -J hops (:932-939)
        for (int t = 0; t < d; t++) h[2 * ((size_t)s * d + t)] -= J * int(one_hop(xs[s] ^ xs[t]));
    // dissipators (init_dissipators :1699-1795)
    for (int c = 0; c < nd; c++) {
        double *lc = l.data() + e2 * c;
        for (int s = 0; s < d; s++) {
            const int b0 = (xs[s] >> c) & 1, b1 = (xs[s] >> (c + 1)) & 1;
            lc[2 * ((size_t)s * d + s)] = diss_type == 0 ? double(b0) : double(b0) - double(b1);
            if (diss_type == 0 || b0 == b1) continue;
            for (int t = 0; t < d; t++) {
                const int g = xs[s] ^ xs[t];
                if (!one_hop(g) || (g & -g) != (1 << c)) continue;  // the pair (c, c+1)
                double *e = lc + 2 * ((size_t)s * d + t);
                e[0] = b0 ? -std::cos(-diss_phase) : std::cos(diss_phase);
                e[1] = b0 ? -std::sin(-diss_phase) : std::sin(diss_phase);
            }
        }
    }
    if (energies) std::memcpy(energies, en.data(), Nc * sizeof(double));
    if (id_to_x) std::memcpy(id_to_x, xs.data(), d * sizeof(int));
    if (H) std::memcpy(H, h.data(), e2 * sizeof(double));
    if (L) std::memcpy(L, l.data(), e2 * nd * sizeof(double));
    if (!Kout && !Utree) return QJX_OK;
    // init_hamiltonians_qj (:2751-2838): H - (i/2) gamma L_c^H L_c added channel by channel, K = -i H_eff
    cvec hp(e2, 0.0), k(e2);
    for (size_t e = 0; e < dd; e++) hp[2 * e] = h[2 * e];
    for (int c = 0; c < nd; c++) {
        const double *lc = l.data() + e2 * c;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                double sr = 0.0, si = 0.0;
                for (int q = 0; q < d; q++) {
                    const double ar = lc[2 * ((size_t)q * d + i)], ai = lc[2 * ((size_t)q * d + i) + 1];
                    const double br = lc[2 * ((size_t)q * d + j)], bi = lc[2 * ((size_t)q * d + j) + 1];
                    sr = sr + (ar * br + ai * bi);
                    si = si + (ar * bi - ai * br);
                }
                const size_t idx = (size_t)i * d + j;
                hp[2 * idx] += 0.5 * (gamma * si);
                hp[2 * idx + 1] -= 0.5 * (gamma * sr);
            }
    }
    for (size_t e = 0; e < dd; e++) {
        k[2 * e] = 0.0 + hp[2 * e + 1];
        k[2 * e + 1] = 0.0 - hp[2 * e];
    }
    if (Kout) std::memcpy(Kout, k.data(), e2 * sizeof(double));
    if (!Utree) return QJX_OK;
    // init_split_structure_mbl (core.cpp:10382-10432): a branch head of duration T whose two
    // children each run the split tree of T (so a period is two T/2 halves of the same K)
    bool ok = true;
#pragma omp parallel for schedule(dynamic, 1) reduction(&& : ok)
    for (int lv = 0; lv < deep; lv++) {
        double dt = T * 0.5;
        for (int q = 0; q <= lv; q++) dt *= 0.5;
        cvec scaled(e2);
        for (size_t e = 0; e < e2; e++) scaled[e] = k[e] * dt;
        ok = expm(d, scaled.data(), Utree + e2 * (size_t)lv) && ok;
    }
    return ok ? QJX_OK : QJX_ERR_INVALID_ARG;
}

// get_imbalance_mbl (source/cpp/QJX/QJX/experiment.cpp:1753-1800) for n rows adr [n][d]: the
// cell occupations n_c = sum_s adr_s n_c(x_s) (s ascending), then (even cells - odd cells) / all.
extern "C" qjx_status qjx_mbl_imbalance(int Nc, int n, const double *adr, double *out)
{
    int d = 0;
    if (qjx_mbl_size(Nc, 0, &d, nullptr) != QJX_OK || n < 0 || (n > 0 && (!adr || !out))) return QJX_ERR_INVALID_ARG;
    const std::vector<int> xs = mbl_words(Nc);
#pragma omp parallel for schedule(static)
    for (int tr = 0; tr < n; tr++) {
        const double *a = adr + (size_t)tr * d;
        std::vector<double> occ(Nc, 0.0);
        for (int s = 0; s < d; s++)
            for (int c = 0; c < Nc; c++) occ[c] += a[s] * double((xs[s] >> (Nc - 1 - c)) & 1);
        double even = 0.0, odd = 0.0;
        for (int c = 0; c < Nc; c++) (c % 2 == 0 ? even : odd) += occ[c];
        const double all = odd + even;
        out[tr] = (even - odd) / all;
    }
    return QJX_OK;
}

// ---------------------------------------------------------------------------------- Integrable
// IntegrableNewDelBehaviour (source/cpp/QJX/QJX/newdel.cpp:310-345, 1030-1095, 1924-2076,
// 2914-3004): N spins (spin 0 the most significant bit of a basis index), d = 2^N, H = 0.
extern "C" qjx_status qjx_build_integrable(int N, int seed, int num_seeds, double tau, double k, double T, int deep,
                                           double *L, double *special, double *Kout, double *Utree)
{
    if (N < 3 || N > 10 || num_seeds < 1 || seed < 0) return QJX_ERR_INVALID_ARG;
    if (Utree && (deep < 1 || !(T > 0.0))) return QJX_ERR_INVALID_ARG;
    const int d = 1 << N;
    const size_t dd = (size_t)d * d, e2 = 2 * dd;
    // channel c < N-1: the 4 x 4 con = tau |00><00| + k |11><11| + |01><10| + |10><01| on spins
    // (c, c+1); channel N-1: the border pair (N-1, 0)
    cvec l(e2 * N, 0.0);
    for (int c = 0; c < N; c++) {
        double *lc = l.data() + e2 * c;
        const int ba = c < N - 1 ? N - 1 - c : 0, bb = c < N - 1 ? N - 2 - c : N - 1;
        for (int s = 0; s < d; s++) {
            const int a = (s >> ba) & 1, b = (s >> bb) & 1;
            if (a == b) lc[2 * ((size_t)s * d + s)] = a ? k : tau;
            else lc[2 * ((size_t)(s ^ (1 << ba) ^ (1 << bb)) * d + s)] = 1.0;
        }
    }
    if (L) std::memcpy(L, l.data(), e2 * N * sizeof(double));
    if (special) {
        // X_ij = g_ij (1 + i), g Box-Muller normals of MCG31 seed 13371337 leapfrogged (seed,
        // num_seeds); y = (X + X^H) / 2, special = y / sqrt(Re tr y^2) / sqrt(d)
        qjxio::LeapfrogLCG st = qjxio::LeapfrogLCG::mcg31(13371337ull, (unsigned long long)seed,
                                                            (unsigned long long)num_seeds);
        const double two_pi = 2.0 * 3.1415926535897932384626433832795;
        std::vector<double> g(dd);
        for (size_t e = 0; e < dd; e++) {
            const double u1 = st.next(), u2 = st.next();
            g[e] = std::sqrt(-2.0 * std::log(u1)) * std::sin(two_pi * u2);
        }
        cvec y(e2);
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                const double gij = g[(size_t)i * d + j], gji = g[(size_t)j * d + i];
                y[2 * ((size_t)i * d + j)] = 0.5 * (gij + gji);
                y[2 * ((size_t)i * d + j) + 1] = 0.5 * (gij + -gji);
            }
        double tr = 0.0;
        for (int i = 0; i < d; i++) {
            double sr = 0.0;
            for (int q = 0; q < d; q++)
                sr = sr + (y[2 * ((size_t)i * d + q)] * y[2 * ((size_t)q * d + i)] -
                           y[2 * ((size_t)i * d + q) + 1] * y[2 * ((size_t)q * d + i) + 1]);
            tr = tr + sr;
        }
        const double sy = std::sqrt(tr), sd = std::sqrt(double(d));
        for (size_t e = 0; e < e2; e++) special[e] = (y[e] / sy) / sd;
    }
    if (!Kout && !Utree) return QJX_OK;
    // init_hamiltonians_qj: H_eff = 0 - (i/2) sum_c L_c^H L_c (gamma 1), K = -i H_eff
    cvec hp(e2, 0.0), kk(e2);
    for (int c = 0; c < N; c++) {
        const double *lc = l.data() + e2 * c;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                double sr = 0.0, si = 0.0;
                for (int q = 0; q < d; q++) {
                    const double ar = lc[2 * ((size_t)q * d + i)], ai = lc[2 * ((size_t)q * d + i) + 1];
                    const double br = lc[2 * ((size_t)q * d + j)], bi = lc[2 * ((size_t)q * d + j) + 1];
                    sr = sr + (ar * br + ai * bi);
                    si = si + (ar * bi - ai * br);
                }
                const size_t idx = (size_t)i * d + j;
                hp[2 * idx] += 0.5 * (1.0 * si);
                hp[2 * idx + 1] -= 0.5 * (1.0 * sr);
            }
    }
    for (size_t e = 0; e < dd; e++) {
        kk[2 * e] = 0.0 + hp[2 * e + 1];
        kk[2 * e + 1] = 0.0 - hp[2 * e];
    }
    if (Kout) std::memcpy(Kout, kk.data(), e2 * sizeof(double));
    if (!Utree) return QJX_OK;
    // init_split_structure_integrable (core.cpp:10610-10660): like MBL, one head of duration T
    // whose two children run the tree of T
    bool ok = true;
#pragma omp parallel for schedule(dynamic, 1) reduction(&& : ok)
    for (int lv = 0; lv < deep; lv++) {
        double dt = T * 0.5;
        for (int q = 0; q <= lv; q++) dt *= 0.5;
        cvec scaled(e2);
        for (size_t e = 0; e < e2; e++) scaled[e] = kk[e] * dt;
        ok = expm(d, scaled.data(), Utree + e2 * (size_t)lv) && ok;
    }
    return ok ? QJX_OK : QJX_ERR_INVALID_ARG;
}

// -------------------------------------------------------------------------------------------- PS
// PSNewDelBehaviour (source/cpp/QJX/QJX/newdel.cpp:132-181, 650-866, 1582-1697, 2603-2749): ns spins
// (spin 0 the most significant bit of the spin index x) times nps photon states; basis index
// x nps + k (Kronecker order spins (x) photons); J = sum of sigma / 2 over the spins.
extern "C" qjx_status qjx_build_ps(int ns, int nps, double alpha, double dprm, double gprm, double drv_ampl,
                                   int diss_type, double diss_w, double part_1, double part_2, int deep, double *H,
                                   double *Hd, double *L, double *S, double *Kout, double *Utree)
{
    if (ns < 1 || ns > 8 || nps < 2 || (diss_type != 0 && diss_type != 1) || !(alpha > 0.0)) return QJX_ERR_INVALID_ARG;
    const int n2 = 1 << ns, d = n2 * nps, nd = diss_type == 0 ? 1 : 1 + ns;
    if (d > 4096) return QJX_ERR_INVALID_ARG;
    if (Utree && (deep < 1 || !(part_1 > 0.0) || !(part_2 > 0.0))) return QJX_ERR_INVALID_ARG;
    const size_t dd = (size_t)d * d, e2 = 2 * dd, pp = (size_t)nps * nps, ss = (size_t)n2 * n2;
    std::vector<double> a(pp, 0.0), ad(pp, 0.0), m1, m2, m3, nop;
    for (int k = 0; k < nps - 1; k++) {
        a[(size_t)k * nps + (k + 1)] = std::sqrt(double(k + 1));
        ad[(size_t)(k + 1) * nps + k] = std::sqrt(double(k + 1));
    }
    real_matmul(nps, ad, ad, m1);
    real_matmul(nps, m1, a, m2);
    real_matmul(nps, m2, a, m3);   // a^+ a^+ a a
    real_matmul(nps, ad, a, nop);  // a^+ a (special_4)
    const double hs = 0.5 / std::pow(alpha, 3);
    // J_z, J_-, J_+ from sigma_z = diag(1, -1), sigma_- = |1><0|, sigma_+ = |0><1| (:700-800)
    std::vector<double> jz(ss, 0.0), jm(ss, 0.0), jp(ss, 0.0);
    for (int sp = 0; sp < ns; sp++)
        for (int x = 0; x < n2; x++) {
            const int bit = 1 << (ns - 1 - sp);
            const bool b = (x & bit) != 0;
            jz[(size_t)x * n2 + x] += b ? -1.0 : 1.0;
            if (!b) jm[(size_t)(x | bit) * n2 + x] += 1.0;
            else jp[(size_t)(x & ~bit) * n2 + x] += 1.0;
        }
    for (size_t e = 0; e < ss; e++) {
        jz[e] *= 0.5;
        jm[e] *= 0.5;
        jp[e] *= 0.5;
    }
    const double sd = dprm * 0.5, sg = gprm * 0.5;
    cvec h(e2, 0.0), hd(e2, 0.0), l(e2 * nd, 0.0), sp4(4 * e2, 0.0);
    for (int xi = 0; xi < n2; xi++)
        for (int xj = 0; xj < n2; xj++)
            for (int ki = 0; ki < nps; ki++)
                for (int kj = 0; kj < nps; kj++) {
                    const size_t e = ((size_t)xi * nps + ki) * d + (size_t)xj * nps + kj;
                    const double id_s = xi == xj ? 1.0 : 0.0, id_p = ki == kj ? 1.0 : 0.0;
                    const size_t pe = (size_t)ki * nps + kj, se = (size_t)xi * n2 + xj;
                    // H = (d/2) J_z (x) 1 + (g/2)(a^+ J_- + J_+ a) + 1 (x) H_photon (:826-833)
                    h[2 * e] = ((sd * jz[se]) * id_p + sg * (ad[pe] * jm[se] + jp[se] * a[pe])) + id_s * (hs * m3[pe]);
                    hd[2 * e] = id_s * (ad[pe] - a[pe]);
                    sp4[2 * e] = id_s * a[pe];
                    sp4[2 * (dd + e)] = jz[se] * id_p;
                    sp4[2 * (2 * dd + e)] = jp[se] * id_p;
                    sp4[2 * (3 * dd + e)] = id_s * nop[pe];
                    l[2 * e] = id_s * a[pe];  // the cavity dissipator 1 (x) a (:1622-1631)
                }
    if (diss_type == 1)  // spin decay sigma_-^(s) (x) 1 (:1633-1695)
        for (int sp = 0; sp < ns; sp++) {
            double *lc = l.data() + e2 * (1 + sp);
            const int bit = 1 << (ns - 1 - sp);
            for (int x = 0; x < n2; x++)
                if (!(x & bit))
                    for (int k = 0; k < nps; k++) lc[2 * (((size_t)(x | bit) * nps + k) * d + (size_t)x * nps + k)] = 1.0;
        }
    if (H) std::memcpy(H, h.data(), e2 * sizeof(double));
    if (Hd) std::memcpy(Hd, hd.data(), e2 * sizeof(double));
    if (L) std::memcpy(L, l.data(), e2 * nd * sizeof(double));
    if (S) std::memcpy(S, sp4.data(), 4 * e2 * sizeof(double));
    if (!Kout && !Utree) return QJX_OK;
    // init_hamiltonians_qj (:2603-2749): gamma 1/(4 alpha) on the cavity, diss_w on the spins;
    // K_0 = -i H_eff + E0 H_drv (the kick), K_1 = -i H_eff
    cvec hp(e2, 0.0);
    for (size_t e = 0; e < dd; e++) hp[2 * e] = h[2 * e];
    for (int c = 0; c < nd; c++) {
        const double *lc = l.data() + e2 * c;
        const double gamma = c == 0 ? 1.0 / (4.0 * alpha) : diss_w;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                double sr = 0.0, si = 0.0;
                for (int q = 0; q < d; q++) {
                    const double ar = lc[2 * ((size_t)q * d + i)], ai = lc[2 * ((size_t)q * d + i) + 1];
                    const double br = lc[2 * ((size_t)q * d + j)], bi = lc[2 * ((size_t)q * d + j) + 1];
                    sr = sr + (ar * br + ai * bi);
                    si = si + (ar * bi - ai * br);
                }
                const size_t idx = (size_t)i * d + j;
                hp[2 * idx] += 0.5 * (gamma * si);
                hp[2 * idx + 1] -= 0.5 * (gamma * sr);
            }
    }
    cvec K[2] = {cvec(e2), cvec(e2)};
    const double Eb[2] = {drv_ampl, 0.0};
    for (size_t e = 0; e < dd; e++)
        for (int b = 0; b < 2; b++) {
            K[b][2 * e] = 0.0 + (hp[2 * e + 1] + Eb[b] * hd[2 * e]);
            K[b][2 * e + 1] = 0.0 - (hp[2 * e] + Eb[b] * 0.0);
        }
    if (Kout) {
        std::memcpy(Kout, K[0].data(), e2 * sizeof(double));
        std::memcpy(Kout + e2, K[1].data(), e2 * sizeof(double));
    }
    if (!Utree) return QJX_OK;
    // init_split_structure_ps (core.cpp:10234-10305): part b's head lasts part_b alpha and runs two
    // children of its tree, each half of it
    const double head[2] = {part_1 * alpha, part_2 * alpha};
    bool ok = true;
#pragma omp parallel for schedule(dynamic, 1) collapse(2) reduction(&& : ok)
    for (int b = 0; b < 2; b++)
        for (int lv = 0; lv < deep; lv++) {
            double dt = head[b] * 0.5;
            for (int q = 0; q <= lv; q++) dt *= 0.5;
            cvec scaled(e2);
            for (size_t e = 0; e < e2; e++) scaled[e] = K[b][e] * dt;
            ok = expm(d, scaled.data(), Utree + e2 * ((size_t)b * deep + lv)) && ok;
        }
    return ok ? QJX_OK : QJX_ERR_INVALID_ARG;
}

// ------------------------------------------------------------------------------------ Floq2Spins
// Floq2SpinsNewDelBehaviour (source/cpp/QJX/QJX/newdel.cpp:346-378, 1096-1182, 2077-2136,
// 3005-3101): two spins (spin 0 the more significant bit), d = 4; the QJ branch is undriven.
extern "C" qjx_status qjx_build_floq2spins(double D1, double D2, double J, double gamma, double T, int deep,
                                           double *H, double *L, double *Kout, double *Utree)
{
    if (Utree && (deep < 1 || !(T > 0.0))) return QJX_ERR_INVALID_ARG;
    const int d = 4;
    const size_t dd = 16, e2 = 32;
    cvec h(e2, 0.0), l(2 * e2, 0.0);
    for (int x = 0; x < d; x++) {  // (Delta_1 sz (x) 1 + Delta_2 1 (x) sz) / 2
        const double s1 = (x & 2) ? -1.0 : 1.0, s2 = (x & 1) ? -1.0 : 1.0;
        h[2 * (x * d + x)] = 0.5 * (D1 * s1 + D2 * s2);
    }
    // J sy (x) sy: anti-diagonal -J, J, J, -J
    h[2 * (0 * d + 3)] = -J;
    h[2 * (1 * d + 2)] = J;
    h[2 * (2 * d + 1)] = J;
    h[2 * (3 * d + 0)] = -J;
    for (int x = 0; x < d; x++) {  // sm (x) 1 and 1 (x) sm, sm = |1><0|
        if (!(x & 2)) l[2 * ((x | 2) * d + x)] = 1.0;
        if (!(x & 1)) l[2 * (dd + (x | 1) * d + x)] = 1.0;
    }
    if (H) std::memcpy(H, h.data(), e2 * sizeof(double));
    if (L) std::memcpy(L, l.data(), 2 * e2 * sizeof(double));
    if (!Kout && !Utree) return QJX_OK;
    cvec hp(h), k(e2);
    for (int c = 0; c < 2; c++) {
        const double *lc = l.data() + e2 * c;
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                double sr = 0.0, si = 0.0;
                for (int q = 0; q < d; q++) {
                    const double ar = lc[2 * (q * d + i)], ai = lc[2 * (q * d + i) + 1];
                    const double br = lc[2 * (q * d + j)], bi = lc[2 * (q * d + j) + 1];
                    sr = sr + (ar * br + ai * bi);
                    si = si + (ar * bi - ai * br);
                }
                hp[2 * (i * d + j)] += 0.5 * (gamma * si);
                hp[2 * (i * d + j) + 1] -= 0.5 * (gamma * sr);
            }
    }
    for (size_t e = 0; e < dd; e++) {
        k[2 * e] = 0.0 + hp[2 * e + 1];
        k[2 * e + 1] = 0.0 - hp[2 * e];
    }
    if (Kout) std::memcpy(Kout, k.data(), e2 * sizeof(double));
    if (!Utree) return QJX_OK;
    // init_split_structure_floq2spins (core.cpp:10722-10766): a head of duration T whose one branch
    // runs the tree of T (so a period advances T / 2)
    bool ok = true;
    for (int lv = 0; lv < deep; lv++) {
        double dt = T * 0.5;
        for (int q = 0; q <= lv; q++) dt *= 0.5;
        cvec scaled(e2);
        for (size_t e = 0; e < e2; e++) scaled[e] = k[e] * dt;
        ok = expm(d, scaled.data(), Utree + e2 * (size_t)lv) && ok;
    }
    return ok ? QJX_OK : QJX_ERR_INVALID_ARG;
}

// -------------------------------------------------------------------------------- FloqManySpins
// FloqManySpinsNewDelBehaviour (source/cpp/QJX/QJX/newdel.cpp:379-413, 1184-1332, 2138-2224,
// 3103-3199): n spins (spin 0 the most significant bit), d = 2^n; the QJ branch is undriven.
extern "C" qjx_status qjx_build_floqnspins(int n, double Delta, double J, double gamma, double T, int deep, double *H,
                                           double *L, double *Kout, double *Utree)
{
    if (n < 1 || n > 10) return QJX_ERR_INVALID_ARG;
    if (Utree && (deep < 1 || !(T > 0.0))) return QJX_ERR_INVALID_ARG;
    const int d = 1 << n;
    const size_t dd = (size_t)d * d, e2 = 2 * dd;
    cvec h(e2, 0.0), l(e2 * n, 0.0);
    const double hd = 0.5 * Delta;
    // i^k for the sy^(x)n entries
    const double ire[4] = {1.0, 0.0, -1.0, 0.0}, iim[4] = {0.0, 1.0, 0.0, -1.0};
    for (int x = 0; x < d; x++) {
        double sz = 0.0;  // sum of the spins' sz (exact integers)
        int z = 0;
        for (int sp = 0; sp < n; sp++) {
            const int b = (x >> (n - 1 - sp)) & 1;
            sz = sz + (b ? -1.0 : 1.0);
            z += !b;
        }
        // n = 1: (Delta / 2) sz; n >= 2: (sum sz) (Delta / 2) + J sy^(x)n, whose only entry in row x
        // is column x ^ (2^n - 1), value i^(n + 2 z) (a factor -i per 0 bit, i per 1 bit)
        h[2 * ((size_t)x * d + x)] = (n == 1) ? hd * sz : sz * hd;
        if (n >= 2) {
            const int k = (n + 2 * z) & 3;
            const size_t e = (size_t)x * d + (x ^ (d - 1));
            h[2 * e] = J * ire[k];
            h[2 * e + 1] = J * iim[k];
        }
        for (int sp = 0; sp < n; sp++) {  // sigma_- = |1><0| on spin sp
            const int bit = 1 << (n - 1 - sp);
            if (!(x & bit)) l[2 * (dd * sp + (size_t)(x | bit) * d + x)] = 1.0;
        }
    }
    if (H) std::memcpy(H, h.data(), e2 * sizeof(double));
    if (L) std::memcpy(L, l.data(), e2 * n * sizeof(double));
    if (!Kout && !Utree) return QJX_OK;
    cvec hp(h), k(e2);
    for (int c = 0; c < n; c++) {
        const double *lc = l.data() + e2 * c;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                double sr = 0.0, si = 0.0;
                for (int q = 0; q < d; q++) {
                    const double ar = lc[2 * ((size_t)q * d + i)], ai = lc[2 * ((size_t)q * d + i) + 1];
                    const double br = lc[2 * ((size_t)q * d + j)], bi = lc[2 * ((size_t)q * d + j) + 1];
                    sr = sr + (ar * br + ai * bi);
                    si = si + (ar * bi - ai * br);
                }
                const size_t idx = (size_t)i * d + j;
                hp[2 * idx] += 0.5 * (gamma * si);
                hp[2 * idx + 1] -= 0.5 * (gamma * sr);
            }
    }
    for (size_t e = 0; e < dd; e++) {
        k[2 * e] = 0.0 + hp[2 * e + 1];
        k[2 * e + 1] = 0.0 - hp[2 * e];
    }
    if (Kout) std::memcpy(Kout, k.data(), e2 * sizeof(double));
    if (!Utree) return QJX_OK;
    // init_split_structure_floqnspins (core.cpp:10825-10871): one branch covering T / 2 per period
    bool ok = true;
#pragma omp parallel for schedule(dynamic, 1) reduction(&& : ok)
    for (int lv = 0; lv < deep; lv++) {
        double dt = T * 0.5;
        for (int q = 0; q <= lv; q++) dt *= 0.5;
        cvec scaled(e2);
        for (size_t e = 0; e < e2; e++) scaled[e] = k[e] * dt;
        ok = expm(d, scaled.data(), Utree + e2 * (size_t)lv) && ok;
    }
    return ok ? QJX_OK : QJX_ERR_INVALID_ARG;
}

// ----------------------------------------------------------------------------------- FloqSpinPh
// FloqSpinPhNewDelBehaviour (source/cpp/QJX/QJX/newdel.cpp:414-449, 1334-1452, 2226-2284, 3201-3297):
// photons (x) spin, basis index 2 k + s, d = 2 (n_ph + 1); the QJ branch is undriven.
extern "C" qjx_status qjx_build_floqspph(int n_ph, double Delta, double Omega, double gamma, double T, int deep,
                                         double *H, double *L, double *Kout, double *Utree)
{
    if (n_ph < 1 || 2 * (n_ph + 1) > 4096) return QJX_ERR_INVALID_ARG;
    if (Utree && (deep < 1 || !(T > 0.0))) return QJX_ERR_INVALID_ARG;
    const int d = 2 * (n_ph + 1);
    const size_t dd = (size_t)d * d, e2 = 2 * dd;
    cvec h(e2, 0.0), l(e2, 0.0);
    const double hd = 0.5 * Delta, ho = 0.5 * Omega;
    for (int k = 0; k <= n_ph; k++) {  // (Delta / 2) 1 (x) sz
        h[2 * ((size_t)(2 * k) * d + 2 * k)] = hd * 1.0;
        h[2 * ((size_t)(2 * k + 1) * d + 2 * k + 1)] = hd * -1.0;
    }
    for (int k = 0; k < n_ph; k++) {
        const double a = std::sqrt(double(k + 1));
        h[2 * ((size_t)(2 * (k + 1) + 1) * d + 2 * k)] = ho * a;  // (Omega / 2) a^+ (x) sm
        h[2 * ((size_t)(2 * k) * d + 2 * (k + 1) + 1)] = ho * a;  // (Omega / 2) a (x) sp
        for (int sp = 0; sp < 2; sp++) l[2 * ((size_t)(2 * k + sp) * d + 2 * (k + 1) + sp)] = a;  // a (x) 1
    }
    if (H) std::memcpy(H, h.data(), e2 * sizeof(double));
    if (L) std::memcpy(L, l.data(), e2 * sizeof(double));
    if (!Kout && !Utree) return QJX_OK;
    cvec hp(h), k(e2);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) {
            double sr = 0.0, si = 0.0;
            for (int q = 0; q < d; q++) {
                const double ar = l[2 * ((size_t)q * d + i)], ai = l[2 * ((size_t)q * d + i) + 1];
                const double br = l[2 * ((size_t)q * d + j)], bi = l[2 * ((size_t)q * d + j) + 1];
                sr = sr + (ar * br + ai * bi);
                si = si + (ar * bi - ai * br);
            }
            const size_t idx = (size_t)i * d + j;
            hp[2 * idx] += 0.5 * (gamma * si);
            hp[2 * idx + 1] -= 0.5 * (gamma * sr);
        }
    for (size_t e = 0; e < dd; e++) {
        k[2 * e] = 0.0 + hp[2 * e + 1];
        k[2 * e + 1] = 0.0 - hp[2 * e];
    }
    if (Kout) std::memcpy(Kout, k.data(), e2 * sizeof(double));
    if (!Utree) return QJX_OK;
    // init_split_structure_flq_sp_ph (core.cpp:10928-10974): one branch covering T / 2 per period
    bool ok = true;
#pragma omp parallel for schedule(dynamic, 1) reduction(&& : ok)
    for (int lv = 0; lv < deep; lv++) {
        double dt = T * 0.5;
        for (int q = 0; q <= lv; q++) dt *= 0.5;
        cvec scaled(e2);
        for (size_t e = 0; e < e2; e++) scaled[e] = k[e] * dt;
        ok = expm(d, scaled.data(), Utree + e2 * (size_t)lv) && ok;
    }
    return ok ? QJX_OK : QJX_ERR_INVALID_ARG;
}
