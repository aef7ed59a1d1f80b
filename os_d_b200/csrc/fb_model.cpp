// fb_model.cpp -- the f-basis Liouvillian of the driven dissipative dimer (host, runs once).
//
// The reference (source/cpp/CQdiss_os_dimer) expands rho = I/d + sum_k x_k F_k in the SU(d)
// generalised Gell-Mann basis (index layout of initRhoODE / calcRho, CQdiss/calcODE.cpp:120-167,
// CQdiss/CalcRho.cpp:4-67: the pairs i < j as (symmetric, antisymmetric), then the d - 1
// diagonal elements) and integrates dx/dt = Gs x + E(t) Qs_drv x - Ks (calcODE.cpp:75-118).  It
// assembles Gs = Qs_base + Rs and Ks from f/d structure-constant tensors (CalcQs.cpp, CalcRs.cpp,
// CalcKs.cpp); the same matrices follow by projection, which is what this file computes:
//
//   Gs_kl = Tr(F_k L0[F_l]),   L0[X] = -i[H_base, X] + gamma (L X L^H - 1/2 {L^H L, X}),
//   Qs_kl = Tr(F_k (-i[H_drv, F_l])),   Ks_k = -Tr(F_k L0[I/d]).
//
// Operators (f-basis conventions, CQdiss/InitH.cpp:227-342, CQdiss/Init_a1_a2.cpp:54-122,
// CQdiss/data.cpp:6-12): H_base = -J hopping, diagonal (2i - N)(-E) + (2i - N)^2 U/N made
// traceless; H_drv = diag(2i - N); L = A1 - i A2 (diag 2i - N, sub-diagonal -sqrt, super +sqrt);
// gamma = g / N.  Every operator is tri- or penta-diagonal and every basis element has at most
// d nonzeros, so each column of Gs is assembled from banded products in O(d) work.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "../../include/qjx_b200.h"

namespace {

using cplx = std::complex<double>;

struct Band {  // sparse rows of a d x d operator
    std::vector<std::vector<std::pair<int, cplx>>> row;
};

struct FbBuilder {
    int N, d, n, npairs;
    double gamma;
    Band Hb, Hd, Lr, Lc, LdL;  // Lc: columns of L as (row, value)
    std::vector<cplx> M;       // d x d scratch
    std::vector<int> touched;
    std::vector<char> mark;

    FbBuilder(int N_, double J, double U, double E, double g)
        : N(N_), d(N_ + 1), n((N_ + 1) * (N_ + 1) - 1), npairs((N_ + 1) * N_ / 2), gamma(g / N_)
    {
        Hb.row.assign(d, {});
        Hd.row.assign(d, {});
        Lr.row.assign(d, {});
        Lc.row.assign(d, {});
        LdL.row.assign(d, {});
        const double Ef = -E, Jf = -J;
        std::vector<double> h2(d);
        double tr = 0.0;
        for (int i = 0; i < d; i++) {
            const double h1 = 2.0 * i - N;
            h2[i] = h1 * Ef + h1 * h1 * U / N;
            tr += h2[i];
        }
        tr /= d;
        for (int i = 0; i < d; i++) {
            if (i > 0) Hb.row[i].push_back({i - 1, Jf * std::sqrt((double)((N - i + 1) * i))});
            Hb.row[i].push_back({i, h2[i] - tr});
            if (i + 1 < d) Hb.row[i].push_back({i + 1, Jf * std::sqrt((double)((N - i) * (i + 1)))});
            Hd.row[i].push_back({i, 2.0 * i - N});
        }
        // L: diag 2i - N, L(i, i+1) = +s_i, L(i+1, i) = -s_i with s_i = sqrt((N - i)(i + 1))
        std::vector<std::vector<cplx>> L(d, std::vector<cplx>(d, 0.0));
        for (int i = 0; i < d; i++) L[i][i] = 2.0 * i - N;
        for (int i = 0; i < N; i++) {
            const double s = std::sqrt((double)((N - i) * (i + 1)));
            L[i][i + 1] = s;
            L[i + 1][i] = -s;
        }
        for (int i = 0; i < d; i++)
            for (int j = std::max(0, i - 1); j <= std::min(d - 1, i + 1); j++)
                if (L[i][j] != 0.0) {
                    Lr.row[i].push_back({j, L[i][j]});
                    Lc.row[j].push_back({i, L[i][j]});
                }
        for (int i = 0; i < d; i++)  // L^H L (penta-diagonal)
            for (int j = std::max(0, i - 2); j <= std::min(d - 1, i + 2); j++) {
                cplx s = 0.0;
                for (int k = std::max(0, std::max(i, j) - 1); k <= std::min(d - 1, std::min(i, j) + 1); k++)
                    s += std::conj(L[k][i]) * L[k][j];
                if (s != 0.0) LdL.row[i].push_back({j, s});
            }
        M.assign((size_t)d * d, 0.0);
        mark.assign((size_t)d * d, 0);
    }

    void add(int i, int j, cplx v)
    {
        const size_t e = (size_t)i * d + j;
        if (!mark[e]) {
            mark[e] = 1;
            touched.push_back((int)e);
        }
        M[e] += v;
    }

    // basis element l as (i, j, value) entries
    void basis(int l, std::vector<std::pair<std::pair<int, int>, cplx>> &F) const
    {
        F.clear();
        const double v = 1.0 / std::sqrt(2.0);
        if (l < 2 * npairs) {
            int p = l / 2, i = 0;
            while (p >= d - 1 - i) {
                p -= d - 1 - i;
                i++;
            }
            const int j = i + 1 + p;
            if ((l & 1) == 0) {
                F.push_back({{i, j}, cplx(v, 0.0)});
                F.push_back({{j, i}, cplx(v, 0.0)});
            } else {
                F.push_back({{i, j}, cplx(0.0, v)});
                F.push_back({{j, i}, cplx(0.0, -v)});
            }
        } else {
            const int m = l - 2 * npairs;
            const double w = 1.0 / std::sqrt((double)((m + 1) * (m + 2)));
            for (int j = 0; j <= m; j++) F.push_back({{j, j}, cplx(w, 0.0)});
            F.push_back({{m + 1, m + 1}, cplx(-(m + 1) * w, 0.0)});
        }
    }

    // M = -i [H, F] + gam (L F L^H - 1/2 {L^H L, F})
    void liou(const Band &H, double gam, const std::vector<std::pair<std::pair<int, int>, cplx>> &F)
    {
        const cplx mi(0.0, -1.0);
        for (const auto &f : F) {
            const int a = f.first.first, b = f.first.second;
            const cplx x = f.second;
            for (const auto &h : H.row[a]) add(h.first, b, mi * h.second * x);   // H F (H symmetric)
            for (const auto &h : H.row[b]) add(a, h.first, -mi * x * h.second);  // -F H
            if (gam != 0.0) {
                for (const auto &li : Lc.row[a])
                    for (const auto &lj : Lc.row[b]) add(li.first, lj.first, gam * li.second * x * std::conj(lj.second));
                for (const auto &q : LdL.row[a]) add(q.first, b, -0.5 * gam * q.second * x);  // L^H L Hermitian
                for (const auto &q : LdL.row[b]) add(a, q.first, -0.5 * gam * x * q.second);
            }
        }
    }

    // f coordinates of M (Tr(F_k M)) as (k, value), then clear the scratch
    void project(std::vector<std::pair<int, double>> &out)
    {
        out.clear();
        const double v = 1.0 / std::sqrt(2.0);
        bool diag = false;
        int dmin = d;
        for (int e : touched) {
            const int i = e / d, j = e % d;
            if (i == j) {
                diag = true;
                dmin = std::min(dmin, i);
                continue;
            }
            if (i > j && mark[(size_t)j * d + i]) continue;  // the pair is visited from (j, i)
            const int a = std::min(i, j), b = std::max(i, j);
            const cplx Mab = M[(size_t)a * d + b], Mba = M[(size_t)b * d + a];
            const int p = a * (2 * d - a - 1) / 2 + (b - a - 1);
            out.push_back({2 * p, (Mab.real() + Mba.real()) * v});
            out.push_back({2 * p + 1, -(Mba.imag() - Mab.imag()) * v});
        }
        if (diag) {
            double s = 0.0;
            for (int m = 0; m < d - 1; m++) {
                s += M[(size_t)m * d + m].real();
                if (m + 1 < dmin) continue;
                const double val = (s - (m + 1) * M[(size_t)(m + 1) * d + (m + 1)].real()) / std::sqrt((double)((m + 1) * (m + 2)));
                out.push_back({2 * npairs + m, val});
            }
        }
        for (int e : touched) {
            M[e] = 0.0;
            mark[e] = 0;
        }
        touched.clear();
    }
};

void to_csr(int n, std::vector<std::vector<std::pair<int, double>>> &rows, double tol, std::vector<int> &rp,
            std::vector<int> &ci, std::vector<double> &v)
{
    rp.assign(n + 1, 0);
    ci.clear();
    v.clear();
    for (int k = 0; k < n; k++) {
        std::vector<std::pair<int, double>> &r = rows[k];
        std::sort(r.begin(), r.end());
        for (size_t e = 0; e < r.size();) {  // merge duplicates, drop rounding residue
            size_t f = e;
            double s = 0.0;
            while (f < r.size() && r[f].first == r[e].first) s += r[f++].second;
            if (std::fabs(s) > tol) {
                ci.push_back(r[e].first);
                v.push_back(s);
            }
            e = f;
        }
        rp[k + 1] = (int)ci.size();
    }
}

}  // namespace

// Liouvillian of the dimer in CSR (rows sorted by column).  Call with null arrays to get the
// nonzero counts, then again with arrays of that size.  Entries whose magnitude is at most
// 1e-14 of the largest entry are rounding residue of exactly-zero elements and are dropped.
extern "C" qjx_status qjx_fb_build_dimer(int N, double J, double U, double E, double g, int *gs_nnz, int *qs_nnz,
                                          int *gs_rowptr, int *gs_col, double *gs_val, int *qs_rowptr,
                                          int *qs_col, double *qs_val, double *Ks)
{
    if (N < 1 || N > 255 || !gs_nnz || !qs_nnz) return QJX_ERR_INVALID_ARG;
    FbBuilder B(N, J, U, E, g);
    const int n = B.n;
    std::vector<std::vector<std::pair<int, double>>> grow(n), qrow(n);
    std::vector<std::pair<std::pair<int, int>, cplx>> F;
    std::vector<std::pair<int, double>> col;
    double gmax = 0.0, qmax = 0.0;
    for (int l = 0; l < n; l++) {
        B.basis(l, F);
        B.liou(B.Hb, B.gamma, F);
        B.project(col);
        for (const auto &c : col) {
            grow[c.first].push_back({l, c.second});
            gmax = std::max(gmax, std::fabs(c.second));
        }
        B.liou(B.Hd, 0.0, F);
        B.project(col);
        for (const auto &c : col) {
            qrow[c.first].push_back({l, c.second});
            qmax = std::max(qmax, std::fabs(c.second));
        }
    }
    std::vector<int> grp, gci, qrp, qci;
    std::vector<double> gv, qv;
    to_csr(n, grow, 1e-14 * gmax, grp, gci, gv);
    to_csr(n, qrow, 1e-14 * qmax, qrp, qci, qv);
    const bool fill = gs_rowptr && gs_col && gs_val && qs_rowptr && qs_col && qs_val && Ks;
    if (fill && (*gs_nnz < (int)gv.size() || *qs_nnz < (int)qv.size())) return QJX_ERR_INVALID_ARG;
    *gs_nnz = (int)gv.size();
    *qs_nnz = (int)qv.size();
    if (!fill) return QJX_OK;
    std::memcpy(gs_rowptr, grp.data(), sizeof(int) * (n + 1));
    std::memcpy(gs_col, gci.data(), sizeof(int) * gci.size());
    std::memcpy(gs_val, gv.data(), sizeof(double) * gv.size());
    std::memcpy(qs_rowptr, qrp.data(), sizeof(int) * (n + 1));
    std::memcpy(qs_col, qci.data(), sizeof(int) * qci.size());
    std::memcpy(qs_val, qv.data(), sizeof(double) * qv.size());
    // Ks = -Tr(F_k L0[I/d])
    F.clear();
    for (int i = 0; i < B.d; i++) F.push_back({{i, i}, cplx(1.0 / B.d, 0.0)});
    B.liou(B.Hb, B.gamma, F);
    B.project(col);
    std::memset(Ks, 0, sizeof(double) * n);
    for (const auto &c : col) Ks[c.first] -= c.second;
    return QJX_OK;
}
