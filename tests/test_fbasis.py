"""The SU(N) f-basis Lindblad solver: oracle checks on CPU, GPU RK4 parity, and the QJ
ensemble against the f-basis density matrix (the density-matrix oracle of the ensemble)."""
import numpy as np
import pytest

from oracle import oracle_py as O
from tests.helpers import T2PI


def dense_rk4(Hb, Hdrv, L, gamma, A, rho, T, num_steps, periods, drv_type=0, freq=1.0, phase=0.0):
    """RK4 of the density matrix with the stage structure of calcODE_trans (calcODE.cpp:278-302)
    and the drive of calcVectValue_real (E(t) = -A sign(sin) or -A sin)."""
    LdL = L.conj().T @ L
    h = T / num_steps

    def f(t, r):
        s = np.sin(freq * t + phase)
        e = -A * s if drv_type == 1 else -A * (-1.0 if s < 0.0 else 1.0)
        Ht = Hb + e * Hdrv
        return (-1j * (Ht @ r - r @ Ht) + gamma * (L @ r @ L.conj().T - 0.5 * (LdL @ r + r @ LdL))) * h

    for p in range(periods):
        for s in range(num_steps):
            t = p * T + s * h
            k1 = f(t, rho)
            k2 = f(t + h / 2, rho + k1 / 2)
            k3 = f(t + h / 2, rho + k2 / 2)
            k4 = f(t + h, rho + k3)
            rho = rho + (k1 + 2 * k2 + 2 * k3 + k4) / 6
    return rho


@pytest.mark.parametrize("N,drv_type,start", [(3, 0, "pure"), (5, 1, "mixed"), (6, 0, "pure")])
def test_fbasis_rk4_equals_dense_density_matrix_rk4(N, drv_type, start):
    J, U, E, A, g = 1.0, 0.5, 1.0, 1.5, 0.4
    Gs, Qs, Ks = O.fb_dense(N, J, U, E, g)
    Hb, Hd, L = O.fb_operators(N, J, U, E)
    d = N + 1
    rho0 = np.zeros((d, d), complex)
    if start == "pure":
        rho0[0, 0] = 1
    else:
        rho0 = np.eye(d) / d
    x0 = O.fb_x_from_rho(N, rho0)
    assert np.allclose(O.fb_rho(N, x0), rho0, atol=1e-15)
    x = O.fb_rk4(O.fb_csr(Gs), O.fb_csr(Qs), Ks, x0, A, drv_type=drv_type, T=T2PI, num_steps=200, n_periods=2)
    rho = dense_rk4(Hb, Hd, L, g / N, A, rho0, T2PI, 200, 2, drv_type=drv_type)
    assert np.abs(O.fb_rho(N, x) - rho).max() < 1e-12
    r = O.fb_rho(N, x)
    assert abs(np.trace(r).real - 1) < 1e-13 and np.allclose(r, r.conj().T, atol=1e-15)


def test_fbasis_operators_match_qjx_operators():
    N, J, U, E = 9, 1.0, 0.5, 1.3
    Hb, Hdrv, Lf = O.fb_operators(N, J, U, E)
    H, Hd, L, K0, K1 = O.dimer_operators(N, J, U, E, 0.0, 0.1)
    # f-basis Hamiltonian = QJX H + E Hd up to a multiple of the identity; H_drv = -Hd; same L
    diff = Hb - (H + E * Hd)
    assert np.allclose(diff - diff[0, 0] * np.eye(N + 1), 0, atol=1e-12)
    assert np.allclose(Hdrv, -Hd) and np.allclose(Lf, L)


def test_liouvillian_structure():
    Gs, Qs, Ks = O.fb_dense(12, 1.0, 0.5, 1.0, 0.1)
    S = O.fb_csr(Gs)
    assert S.nnz < 0.1 * Gs.size  # sparse
    # the drive commutator only couples the coherences of each pair (i, j): 2 x 2 blocks
    assert np.abs(np.diag(Qs)).max() == 0.0
    assert np.count_nonzero(Qs) == 12 * 13


def test_qj_ensemble_within_statistical_error_of_fbasis_rho():
    N, n, periods = 4, 3000, 3
    J, U, E, A, g = 1.0, 0.5, 1.0, 1.5, 2.0
    Gs, Qs, Ks = O.fb_dense(N, J, U, E, g)
    rho0 = np.zeros((N + 1, N + 1), complex)
    rho0[0, 0] = 1
    x = O.fb_x_from_rho(N, rho0)
    H, Hd, L, K0, K1 = O.dimer_operators(N, J, U, E, A, g)
    Ut = np.stack([O.split_tree(K0, T2PI, 16), O.split_tree(K1, T2PI, 16)])
    ens = O.Ensemble(Ut, L, [1.0], H + E * Hd, None, T2PI, n, seed=9, record=0)
    ens.init(0, 0)
    Gc, Qc = O.fb_csr(Gs), O.fb_csr(Qs)
    for p in range(periods):
        x = O.fb_rk4(Gc, Qc, Ks, x, A, T=T2PI, num_steps=2000, period0=p, n_periods=1)
        assert ens.run_periods(1) == 0
        pops_f = np.real(np.diag(O.fb_rho(N, x)))
        adr = ens.observables(want_adr=True)["adr"]
        err = adr.std(axis=0) / np.sqrt(n)
        assert np.all(np.abs(adr.mean(axis=0) - pops_f) < 4.5 * err + 2e-3), (adr.mean(axis=0), pops_f)


@pytest.mark.gpu
@pytest.mark.parametrize("N,drv_type", [(5, 0), (20, 0), (20, 1)])
def test_gpu_rk4_matches_oracle(N, drv_type):
    import os_d_b200 as q

    Gs, Qs, Ks = O.fb_dense(N, 1.0, 0.5, 1.0, 0.1)
    Gc, Qc = O.fb_csr(Gs), O.fb_csr(Qs)
    rho0 = np.zeros((N + 1, N + 1), complex)
    rho0[0, 0] = 1
    x0 = O.fb_x_from_rho(N, rho0)
    steps, periods = 300, 2
    x_o = O.fb_rk4(Gc, Qc, Ks, x0, 1.5, drv_type=drv_type, T=T2PI, num_steps=steps, n_periods=periods)
    fb = q.FBasis(Gc, Qc, Ks, x0, 1.5, drv_type=drv_type, T=T2PI, num_steps=steps)
    fb.run(0, periods)
    x_g, _ = fb.get()
    if drv_type == 0:
        assert np.array_equal(x_g, x_o)  # sign of sin only: bit-exact
    else:
        assert np.abs(x_g - x_o).max() < 1e-12  # CUDA sin vs libm sin
    fb.close()


@pytest.mark.gpu
def test_gpu_qj_ensemble_within_statistical_error_of_gpu_fbasis():
    import os_d_b200 as q

    N, n, periods = 12, 6000, 2
    J, U, E, A, g = 1.0, 0.5, 1.0, 1.5, 1.0
    Gs, Qs, Ks = O.fb_dense(N, J, U, E, g)
    rho0 = np.zeros((N + 1, N + 1), complex)
    rho0[0, 0] = 1
    fb = q.FBasis(O.fb_csr(Gs), O.fb_csr(Qs), Ks, O.fb_x_from_rho(N, rho0), A, T=T2PI, num_steps=2000)
    H, Hd, L, Ut = q.build_dimer(N, J, U, E, A, g, 1.0, 16)
    eng = q.Engine(Ut, L, [1.0], H + E * Hd, None, T2PI, n, seed=21, max_dumps=periods + 1, keep_adr=1)
    psi0 = np.zeros((n, N + 1), complex)
    psi0[:, 0] = 1
    eng.set_states(psi0)
    eng.init_thresholds()
    eng.run_periods(periods, dump_at=list(range(1, periods + 1)), dump_base=1)
    adr = eng.observables(1, periods, want_adr=True)["adr"]
    for p in range(periods):
        fb.run(p, 1)
        x, _ = fb.get()
        pops_f = np.real(np.diag(O.fb_rho(N, x)))
        err = adr[p].std(axis=0) / np.sqrt(n)
        assert np.all(np.abs(adr[p].mean(axis=0) - pops_f) < 4.5 * err + 2e-3)


@pytest.mark.gpu
@pytest.mark.parametrize("N", [20, 50])
def test_gpu_cluster_rk4_matches_oracle_and_stage_kernels(N, monkeypatch):
    import os_d_b200 as q

    Gs, Qs, Ks = O.fb_dense(N, 1.0, 0.5, 1.0, 0.1)
    Gc, Qc = O.fb_csr(Gs), O.fb_csr(Qs)
    rho0 = np.zeros((N + 1, N + 1), complex)
    rho0[0, 0] = 1
    x0 = O.fb_x_from_rho(N, rho0)
    steps = 200 if N == 20 else 2000  # RK4 stability: h times the spectral radius of Gs stays < 2.5
    fb = q.FBasis(Gc, Qc, Ks, x0, 1.5, drv_type=0, T=T2PI, num_steps=steps)
    assert fb.cluster_size() > 0  # the cluster-resident path is taken
    fb.run(0, 2)
    x_c, _ = fb.get()
    monkeypatch.setenv("QJX_FB_PATH", "stages")
    fs = q.FBasis(Gc, Qc, Ks, x0, 1.5, drv_type=0, T=T2PI, num_steps=steps)
    assert fs.cluster_size() == 0
    fs.run(0, 2)
    x_s, _ = fs.get()
    assert np.all(np.isfinite(x_c)) and np.array_equal(x_c, x_s)
    x_o = O.fb_rk4(Gc, Qc, Ks, x0, 1.5, drv_type=0, T=T2PI, num_steps=steps, n_periods=2)
    assert np.array_equal(x_c, x_o)


def _fb_system(N):
    """CSR Gs, Qs_drv and Ks of the dimer from the library's builder (the oracle's dense projection
    would hold n^2 doubles at these sizes), as scipy matrices for the oracle's RK4."""
    import scipy.sparse as sp

    from os_d_b200 import _native as Nt

    (gr, gc, gv), (qr, qc, qv), ks = Nt.fb_build_dimer(N, 1.0, 0.5, 1.0, 0.1)
    n = (N + 1) ** 2 - 1
    return sp.csr_matrix((gv, gc, gr), shape=(n, n)), sp.csr_matrix((qv, qc, qr), shape=(n, n)), ks


@pytest.mark.gpu
def test_gpu_stage_kernels_beyond_the_cluster_match_oracle_and_repeat(monkeypatch):
    """N = 100 (n = 10,200) does not fit the cluster-resident path: the per-stage kernels, whose
    rows read other rows' stage arguments, run over 8,400 blocks that cannot all be resident at
    once.  60 RK4 steps across a sign change of the drive equal the oracle bit for bit, twice."""
    import os_d_b200 as q

    N = 100
    Gc, Qc, Ks = _fb_system(N)
    x0 = q.fbasis_pure_state(N, 0)
    steps, T, period0 = 60, 0.24, 12  # t in [2.88, 3.12] and [3.12, 3.36]: sign(sin t) flips at pi
    monkeypatch.setenv("QJX_FB_PATH", "stages")
    runs = []
    for _ in range(2):
        fb = q.FBasis(Gc, Qc, Ks, x0, 1.5, drv_type=0, T=T, num_steps=steps)
        assert fb.cluster_size() == 0
        fb.run(period0, 2)
        runs.append(fb.get()[0])
        fb.close()
    x_o = O.fb_rk4(Gc, Qc, Ks, x0, 1.5, drv_type=0, T=T, num_steps=steps, period0=period0, n_periods=2)
    assert np.all(np.isfinite(x_o)) and np.abs(x_o - x0).max() > 1e-6
    assert np.array_equal(runs[0], x_o)
    assert np.array_equal(runs[1], x_o)


@pytest.mark.gpu
def test_qj_ensemble_at_d51_within_3_sigma_of_fbasis_rho():
    """The f-basis steady-state check: dimer N = 50 (d = 51; J 1, U 0.5, E 1, A 1.5, g 0.1), the QJ
    ensemble of 10^4 trajectories from |N,0> against the f-basis density matrix from the same state (Liouvillian from
    the library's builder, RK4 with dt = 1e-3: 6284 steps per period), both on the GPU.  After 40
    periods (the periodic steady state: the populations change by less than their statistical error
    between the last two dumps) every one of the 51 populations lies within 3 standard errors of the
    ensemble estimate, with no absolute slack."""
    import math

    import os_d_b200 as q

    N, n, J, U, E, A, g = 50, 10000, 1.0, 0.5, 1.0, 1.5, 0.1
    dumps = [10, 20, 30, 40]
    Gc, Qc, Ks = _fb_system(N)
    steps = math.ceil(T2PI / 1e-3)
    fb = q.FBasis(Gc, Qc, Ks, q.fbasis_pure_state(N, 0), A, T=T2PI, num_steps=steps)
    H, Hd, L, Ut = q.build_dimer(N, J, U, E, A, g, 1.0, 16)
    eng = q.Engine(Ut, L, [1.0], H + E * Hd, None, T2PI, n, seed=7, max_dumps=len(dumps) + 1, keep_adr=1)
    psi0 = np.zeros((n, N + 1), complex)
    psi0[:, 0] = 1
    eng.set_states(psi0)
    eng.init_thresholds()
    eng.run_periods(dumps[-1], dump_at=dumps, dump_base=1)
    adr = eng.observables(1, len(dumps), want_adr=True)["adr"]
    eng.close()
    zmax, done = [], 0
    for i, p in enumerate(dumps):
        fb.run(done, p - done)
        done = p
        pops_f = np.real(np.diag(O.fb_rho(N, fb.get()[0])))
        est, err = adr[i].mean(axis=0), adr[i].std(axis=0) / np.sqrt(n)
        assert np.all(err > 0)
        zmax.append(float(np.abs((est - pops_f) / err).max()))
    fb.close()
    print("max |z| per dump (periods %s): %s" % (dumps, zmax))
    last = adr[-1].mean(axis=0) - adr[-2].mean(axis=0)
    assert np.all(np.abs(last) < 3 * np.hypot(adr[-1].std(axis=0), adr[-2].std(axis=0)) / np.sqrt(n))
    assert zmax[-1] <= 3.0
