// fbasis_ref_driver.cpp -- C entry points over the reference's own f-basis Lindblad code
// (source/cpp/CQdiss_os_dimer), compiled unmodified from the reference tree by oracle/build_ref.py
// into oracle/_ref/libfbref.so.  Test infrastructure only: it pins the f-basis oracle and the
// library's Liouvillian builder to what the reference itself assembles and integrates.
//
// The flow is the reference's f_basis_prop_std (CQdiss/data.cpp:18-50): init_main_data (T = 2 pi,
// step = T / num_steps, diss_gamma /= N), createModel, f_basis_init (CQdiss/f_basis_init.cpp:11-104:
// operators, Qs_base, Qs_drv, Ks, Rs, Gs = Qs_base + Rs, initRhoODE), then calcODE_trans
// (CQdiss/calcODE.cpp:249-309) for the RK4 periods.  The initial state is the pure state
// |int_isi><int_isi| (init_conditions, calcODE.cpp:4-33 with int_ist 0).
#include <cmath>
#include <cstring>
#include <iostream>

#include "Model.h"
#include "calcODE.h"
#include "data.h"
#include "f_basis_init.h"

namespace {

Model *build(int N, double J, double U, double E, double g, int drv_type, double A, int num_steps, int start_state,
             RunParam &rp, ConfigParam &cp, MainData &md)
{
    cp = ConfigParam();
    cp.N = N;
    cp.prm_J = J;
    cp.prm_U = U;
    cp.prm_E = E;
    cp.diss_type = 0;
    cp.diss_gamma = g;
    cp.diss_phase = 0.0;
    cp.drv_type = drv_type;
    cp.drv_ampl = A;
    cp.drv_freq = 1.0;
    cp.drv_phase = 0.0;
    cp.num_steps = num_steps;
    cp.int_ist = 0;
    cp.int_isi = start_state;
    rp = RunParam();
    std::streambuf *old = std::cout.rdbuf(nullptr);  // the reference prints its stage timings
    init_main_data(rp, cp, md);
    Model *m = createModel(md.size - 1, cp);
    f_basis_init(m, rp, cp, md);
    std::cout.rdbuf(old);
    std::cout.clear();
    return m;
}

void export_csr(const crsMatrix *M, int *rowptr, int *col, double *val, double *max_imag)
{
    for (int i = 0; i <= M->N; i++) rowptr[i] = M->RowIndex[i];
    for (int p = 0; p < M->NZ; p++) {
        col[p] = M->Col[p];
        val[p] = M->Value[p].re;
        *max_imag = std::fmax(*max_imag, std::fabs(M->Value[p].im));
    }
}

}  // namespace

// Gs, Qs_drv (zero-based CSR as the reference stores them after assembly), Ks and the initial
// f-vector RhoF of the dimer.  Call with null arrays for the nonzero counts, then with arrays of
// those sizes (row pointers (N+1)^2).  *max_imag receives the largest imaginary part the reference
// left in Gs, Qs_drv, Ks and RhoF (the f-basis problem is real).
extern "C" int fbref_build(int N, double J, double U, double E, double g, int start_state, int *gs_nnz, int *qs_nnz,
                           int *gs_rowptr, int *gs_col, double *gs_val, int *qs_rowptr, int *qs_col, double *qs_val,
                           double *Ks, double *x0, double *max_imag)
{
    if (N < 1 || start_state < 0 || start_state > N || !gs_nnz || !qs_nnz) return 1;
    RunParam rp;
    ConfigParam cp;
    MainData md;
    Model *m = build(N, J, U, E, g, 0, 0.0, 1000, start_state, rp, cp, md);
    *gs_nnz = m->Gs->NZ;
    *qs_nnz = m->Qs_drv->NZ;
    if (gs_rowptr) {
        double mi = 0.0;
        export_csr(m->Gs, gs_rowptr, gs_col, gs_val, &mi);
        export_csr(m->Qs_drv, qs_rowptr, qs_col, qs_val, &mi);
        for (int i = 0; i < m->N_mat; i++) {
            Ks[i] = m->Ks[i].re;
            x0[i] = m->RhoF[i].re;
            mi = std::fmax(mi, std::fmax(std::fabs(m->Ks[i].im), std::fabs(m->RhoF[i].im)));
        }
        if (max_imag) *max_imag = mi;
    }
    freeModel(m);
    return 0;
}

// The reference's RK4 (calcODE_trans) over n_periods periods of num_steps steps from the pure
// state |start_state>, drive type drv_type (0: -A sign(sin t), 1: -A sin t); x receives RhoF.
extern "C" int fbref_rk4(int N, double J, double U, double E, double g, int drv_type, double A, int num_steps,
                         int n_periods, int start_state, double *x)
{
    if (N < 1 || num_steps < 1 || n_periods < 0 || !x) return 1;
    RunParam rp;
    ConfigParam cp;
    MainData md;
    Model *m = build(N, J, U, E, g, drv_type, A, num_steps, start_state, rp, cp, md);
    const int n = m->N_mat;
    PropData pd;
    std::memset(&pd, 0, sizeof(pd));
    pd.k1 = new double[n];
    pd.k2 = new double[n];
    pd.k3 = new double[n];
    pd.k4 = new double[n];
    pd.val = new double[n];
    pd.tmp = new double[n];
    pd.tmp_drv = new double[n];
    cp.num_periods_trans = n_periods;
    calcODE_trans(m, rp, cp, md, pd);
    for (int i = 0; i < n; i++) x[i] = m->RhoF[i].re;
    delete[] pd.k1;
    delete[] pd.k2;
    delete[] pd.k3;
    delete[] pd.k4;
    delete[] pd.val;
    delete[] pd.tmp;
    delete[] pd.tmp_drv;
    freeModel(m);
    return 0;
}
