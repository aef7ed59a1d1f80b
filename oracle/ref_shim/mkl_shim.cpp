// mkl_shim.cpp -- CSR kernels with the documented semantics of the MKL routines declared in
// mkl.h (test infrastructure for the f-basis oracle pin, see oracle/build_ref.py).
//
// Choices where the documentation leaves the order open: every output row lists its columns in
// ascending order (a valid CSR whatever the input order), entries repeated within an input row add
// up, an entry of C = A + beta B present in both operands is a + beta b, and a product entry sums
// its terms in the order of A's row.  The
// `sort` argument (reordering of the inputs) is honoured by sorting a copy of each input row.
#include "mkl.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <utility>
#include <vector>

namespace {

using Row = std::vector<std::pair<int, MKL_Complex16>>;  // (zero-based column, value)

MKL_Complex16 cadd(MKL_Complex16 x, MKL_Complex16 y) { return {x.real + y.real, x.imag + y.imag}; }
MKL_Complex16 cmul(MKL_Complex16 x, MKL_Complex16 y)
{
    return {x.real * y.real - x.imag * y.imag, x.real * y.imag + x.imag * y.real};
}
MKL_Complex16 cconj(MKL_Complex16 x) { return {x.real, -x.imag}; }

// One-based CSR (rows x cols) into zero-based rows; op 'T' / 'C' transposes (and conjugates).
std::vector<Row> rows_of(const MKL_Complex16 *v, const int *ja, const int *ia, int rows, int cols, char op, bool sort_in)
{
    const bool tr = (op == 'T' || op == 't' || op == 'C' || op == 'c');
    const bool cj = (op == 'C' || op == 'c');
    std::vector<Row> out(tr ? cols : rows);
    for (int i = 0; i < rows; i++) {
        Row r;
        for (int p = ia[i] - 1; p < ia[i + 1] - 1; p++) r.push_back({ja[p] - 1, v[p]});
        if (sort_in)
            std::stable_sort(r.begin(), r.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
        for (const auto &e : r) {
            if (tr) out[e.first].push_back({i, cj ? cconj(e.second) : e.second});
            else out[i].push_back(e);
        }
    }
    return out;
}

// Writes rows into one-based CSR according to `request`; returns the info code.
int emit(const std::vector<Row> &C, int request, MKL_Complex16 *c, int *jc, int *ic, const int *nzmax)
{
    const int m = (int)C.size();
    if (request == 1 || request == 0) {
        ic[0] = 1;
        for (int i = 0; i < m; i++) ic[i + 1] = ic[i] + (int)C[i].size();
        if (request == 1) return 0;
    }
    for (int i = 0; i < m; i++) {
        int p = ic[i] - 1;
        for (const auto &e : C[i]) {
            if (request == 0 && nzmax && p >= *nzmax) return i + 1;
            jc[p] = e.first + 1;
            c[p] = e.second;
            p++;
        }
    }
    return 0;
}

Row sorted_row(const std::map<int, MKL_Complex16> &acc)
{
    Row r;
    for (const auto &kv : acc) r.push_back(kv);
    return r;
}

}  // namespace

extern "C" void mkl_dcsrgemv(const char *transa, const int *m, const double *a, const int *ia, const int *ja,
                             const double *x, double *y)
{
    const int n = *m;
    const char t = *transa;
    if (t == 'N' || t == 'n') {
        for (int i = 0; i < n; i++) {
            double s = 0.0;
            for (int p = ia[i] - 1; p < ia[i + 1] - 1; p++) s += a[p] * x[ja[p] - 1];
            y[i] = s;
        }
        return;
    }
    for (int i = 0; i < n; i++) y[i] = 0.0;
    for (int i = 0; i < n; i++)
        for (int p = ia[i] - 1; p < ia[i + 1] - 1; p++) y[ja[p] - 1] += a[p] * x[i];
}

extern "C" void mkl_zcsradd(const char *trans, const int *request, const int *sort, const int *m, const int *n,
                            MKL_Complex16 *a, int *ja, int *ia, MKL_Complex16 *beta, MKL_Complex16 *b, int *jb,
                            int *ib, MKL_Complex16 *c, int *jc, int *ic, const int *nzmax, int *info)
{
    const int s = *sort;
    const std::vector<Row> A = rows_of(a, ja, ia, *m, *n, 'N', s == 1 || s == 3);
    const char op = *trans;
    const bool tr = (op == 'T' || op == 't' || op == 'C' || op == 'c');
    const std::vector<Row> B = rows_of(b, jb, ib, tr ? *n : *m, tr ? *m : *n, op, s == 2 || s == 3);
    std::vector<Row> C(*m);
    for (int i = 0; i < *m; i++) {
        std::map<int, MKL_Complex16> acc;  // entries repeated within a row add up
        for (const auto &e : A[i]) {
            auto it = acc.find(e.first);
            if (it == acc.end()) acc[e.first] = e.second;
            else it->second = cadd(it->second, e.second);
        }
        for (const auto &e : B[i]) {
            const MKL_Complex16 v = cmul(*beta, e.second);
            auto it = acc.find(e.first);
            if (it == acc.end()) acc[e.first] = v;
            else it->second = cadd(it->second, v);
        }
        C[i] = sorted_row(acc);
    }
    *info = emit(C, *request, c, jc, ic, nzmax);
}

extern "C" void mkl_zcsrmultcsr(const char *trans, const int *request, const int *sort, const int *m, const int *n,
                                const int *k, MKL_Complex16 *a, int *ja, int *ia, MKL_Complex16 *b, int *jb, int *ib,
                                MKL_Complex16 *c, int *jc, int *ic, const int *nzmax, int *info)
{
    const int s = *sort;
    const char op = *trans;
    const bool tr = (op == 'T' || op == 't' || op == 'C' || op == 'c');
    const std::vector<Row> A = rows_of(a, ja, ia, *m, *n, op, s == 1 || s == 3);  // rows of op(A)
    const std::vector<Row> B = rows_of(b, jb, ib, tr ? *m : *n, *k, 'N', s == 2 || s == 3);
    std::vector<Row> C(A.size());
    for (size_t i = 0; i < A.size(); i++) {
        std::map<int, MKL_Complex16> acc;
        for (const auto &ea : A[i])
            for (const auto &eb : B[ea.first]) {
                const MKL_Complex16 v = cmul(ea.second, eb.second);
                auto it = acc.find(eb.first);
                if (it == acc.end()) acc[eb.first] = v;
                else it->second = cadd(it->second, v);
            }
        C[i] = sorted_row(acc);
    }
    *info = emit(C, *request, c, jc, ic, nzmax);
}

extern "C" lapack_int LAPACKE_zgeev(int, char, char, lapack_int, MKL_Complex16 *, lapack_int, MKL_Complex16 *,
                                    MKL_Complex16 *, lapack_int, MKL_Complex16 *, lapack_int)
{
    std::fprintf(stderr, "LAPACKE_zgeev is not available in the oracle shim (Floquet tasks only)\n");
    return -1;
}
