"""ctypes bindings of the CPU oracle (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module; the product (os_d_b200) never does.
"""
import ctypes as C
import os

import numpy as np

from . import build_oracle

_lib = None

c_double_p = C.POINTER(C.c_double)
c_int_p = C.POINTER(C.c_int)
c_i64_p = C.POINTER(C.c_int64)


class OrcProblem(C.Structure):
    _fields_ = [("d", C.c_int), ("n_traj", C.c_int), ("deep", C.c_int), ("num_branches", C.c_int),
                ("num_diss", C.c_int), ("num_robs", C.c_int), ("record", C.c_int), ("rng_kind", C.c_int),
                ("T", C.c_double), ("seed", C.c_uint64),
                ("U", c_double_p), ("L", c_double_p), ("g", c_double_p), ("HE", c_double_p), ("R", c_double_p),
                ("inj_u", c_double_p), ("inj_off", c_i64_p), ("tr_base", C.c_uint64), ("branch_len", c_double_p)]


class OrcState(C.Structure):
    _fields_ = [("phi", c_double_p), ("eta", c_double_p), ("t", c_double_p), ("rng_pos", c_i64_p),
                ("jumps_counts", c_int_p), ("matvecs", c_i64_p), ("rec_cap", C.c_int), ("n_rec", c_int_p),
                ("jump_times", c_double_p), ("jump_norms", c_double_p), ("jump_etas", c_double_p),
                ("diss_types", c_int_p), ("error", c_int_p), ("rng_src", c_int_p)]


class OrcLpnConfig(C.Structure):
    _fields_ = [("lpn_type", C.c_int), ("eps_deep", C.c_int), ("per_period", C.c_int), ("pad", C.c_int),
                ("eps_low", C.c_double), ("eps_high", C.c_double), ("eps_error", C.c_double),
                ("delta_s", C.c_double), ("delta_f_high", C.c_double), ("delta_f_low", C.c_double),
                ("max_energy", C.c_double), ("mbl_Nc", C.c_int), ("chars_sys", C.c_int), ("spec_div", C.c_double)]


class OrcLpn(C.Structure):
    _fields_ = [("lambda_", c_double_p), ("lambda_now", c_double_p), ("delta_s", c_double_p),
                ("mean_lpn", c_double_p), ("energy_lpn", c_double_p), ("robs_lpn", c_double_p),
                ("num_renorms", c_int_p), ("var_pos", c_i64_p), ("renormed", c_int_p), ("ratio", c_double_p),
                ("ds_rec", c_double_p), ("df_rec", c_double_p), ("eps_iters", c_int_p), ("eps", c_double_p)]


class OrcRk(C.Structure):
    _fields_ = [("ND", c_double_p), ("DR", c_double_p), ("E0", C.c_double), ("A", C.c_double), ("freq", C.c_double),
                ("phase", C.c_double), ("drv_type", C.c_int), ("rk_ns", C.c_int)]


def lib():
    global _lib
    if _lib is None:
        path = build_oracle.build()
        _lib = C.CDLL(path)
        L = _lib
        L.orc_dimer_operators.argtypes = [C.c_int] + [C.c_double] * 5 + [c_double_p] * 5
        L.orc_expm.argtypes = [C.c_int, c_double_p, c_double_p]
        L.orc_dimer_heff.argtypes = [C.c_int] + [C.c_double] * 4 + [c_double_p]
        L.orc_jcs_operators.argtypes = [C.c_int, C.c_double, C.c_double] + [c_double_p] * 6
        L.orc_mbl_basis.argtypes = [C.c_int, c_int_p]
        L.orc_mcg31_uniform.argtypes = [C.c_ulonglong] * 3 + [C.c_int, C.c_double, C.c_double, c_double_p]
        L.orc_mbl_operators.argtypes = ([C.c_int] + [C.c_double] * 3 + [C.c_int] * 3 + [C.c_double] * 2
                                        + [c_double_p] * 4)
        L.orc_mbl_imbalance.argtypes = [C.c_int, C.c_int, C.c_int, c_double_p, c_double_p]
        L.orc_ps_operators.argtypes = [C.c_int] * 2 + [C.c_double] * 4 + [C.c_int, C.c_double] + [c_double_p] * 6
        L.orc_floq2spins_operators.argtypes = [C.c_double] * 4 + [c_double_p] * 3
        L.orc_floqnspins_operators.argtypes = [C.c_int] + [C.c_double] * 3 + [c_double_p] * 3
        L.orc_floqspph_operators.argtypes = [C.c_int] + [C.c_double] * 3 + [c_double_p] * 3
        L.orc_integrable_operators.argtypes = [C.c_int] * 3 + [C.c_double] * 2 + [c_double_p] * 3
        L.orc_split_tree.argtypes = [C.c_int, c_double_p, C.c_double, C.c_int, c_double_p]
        L.orc_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_philox_uniform.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.orc_philox_uniform.restype = C.c_double
        L.orc_init.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcState), C.c_int, C.c_int]
        L.orc_run_branch_units.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcState)] + [C.c_int] * 6
        L.orc_run_periods_rk.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcRk), C.POINTER(OrcState), C.c_int,
                                         C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_run_periods.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcState), C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_int]
        L.orc_observables.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcState), C.c_int] + [c_double_p] * 8
        L.orc_dump_periods.argtypes = [C.c_int, C.c_int, C.c_int, c_int_p]
        L.orc_lpn_start.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcState), C.POINTER(OrcLpnConfig),
                                    C.POINTER(OrcLpn)]
        L.orc_lpn_period.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcState), C.POINTER(OrcLpnConfig),
                                     C.POINTER(OrcLpn), C.c_double]
        L.orc_lpn_bases.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcState), C.POINTER(OrcLpnConfig),
                                    C.POINTER(OrcLpn)]
        L.orc_lpn_exp10.argtypes = [C.c_double]
        L.orc_lpn_exp10.restype = C.c_double
        L.orc_lpn_log.argtypes = [C.c_double]
        L.orc_lpn_log.restype = C.c_double
        L.orc_matvec.argtypes = [C.c_int, c_double_p, c_double_p, c_double_p]
        L.orc_norm_square.argtypes = [C.c_int, c_double_p]
        L.orc_norm_square.restype = C.c_double
        L.orc_purity.argtypes = [C.c_int, C.c_int, c_double_p, c_double_p]
        L.orc_purity.restype = C.c_double
    return _lib


def _dp(a):
    return a.ctypes.data_as(c_double_p) if a is not None else None


def _cplx(shape):
    return np.zeros(shape, dtype=np.complex128)


def dimer_operators(N, J, U, E, A, g):
    d = N + 1
    H, Hd, L, K0, K1 = (_cplx((d, d)) for _ in range(5))
    rc = lib().orc_dimer_operators(N, J, U, E, A, g, _dp(H), _dp(Hd), _dp(L), _dp(K0), _dp(K1))
    assert rc == 0
    return H, Hd, L, K0, K1


def jcs_operators(N, alpha, drv_ampl):
    """JCS (sys_id 1): H, H_drv, L = a, Nop = a^+ a, K0, K1 (d = N)."""
    d = N
    out = [_cplx((d, d)) for _ in range(6)]
    assert lib().orc_jcs_operators(N, alpha, drv_ampl, *[_dp(x) for x in out]) == 0
    return tuple(out)


def mbl_basis(Nc):
    """The MBL basis words (Nc/2 of Nc bits set, ascending)."""
    d = lib().orc_mbl_basis(Nc, None)
    assert d > 0
    xs = np.zeros(d, dtype=np.int32)
    lib().orc_mbl_basis(Nc, xs.ctypes.data_as(c_int_p))
    return xs


def mcg31_uniform(seed, k, s, count, a, b):
    out = np.zeros(count)
    lib().orc_mcg31_uniform(seed, k, s, count, a, b, _dp(out))
    return out


def mbl_operators(Nc, W, U, J, mbl_seed, mbl_mns, diss_type, diss_phase, gamma):
    """MBL (sys_id 3): energies [Nc], H, L [num_diss], K = hamiltonians_qj[0] (d = C(Nc, Nc/2))."""
    d = len(mbl_basis(Nc))
    nd = Nc if diss_type == 0 else Nc - 1
    en = np.zeros(Nc)
    H, K = _cplx((d, d)), _cplx((d, d))
    L = _cplx((nd, d, d))
    assert lib().orc_mbl_operators(Nc, W, U, J, mbl_seed, mbl_mns, diss_type, diss_phase, gamma, _dp(en), _dp(H),
                                   _dp(L), _dp(K)) == 0
    return en, H, L, K


def ps_operators(ns, nps, alpha, dprm, gprm, drv_ampl, diss_type, diss_w):
    """PS (sys_id 2): H, Hd, L [1 + ns diss_type], S [4] (spec, spec_2, spec_3, photons), K0, K1."""
    d = (1 << ns) * nps
    nd = 1 if diss_type == 0 else 1 + ns
    H, Hd, K0, K1 = (_cplx((d, d)) for _ in range(4))
    L, S = _cplx((nd, d, d)), _cplx((4, d, d))
    assert lib().orc_ps_operators(ns, nps, alpha, dprm, gprm, drv_ampl, diss_type, diss_w, _dp(H), _dp(Hd), _dp(L),
                                  _dp(S), _dp(K0), _dp(K1)) == 0
    return H, Hd, L, S, K0, K1


def floq2spins_operators(D1, D2, J, gamma):
    """Floq2Spins (sys_id 7): H (= special), L [2], K = hamiltonians_qj[0] (d = 4)."""
    H, K, L = _cplx((4, 4)), _cplx((4, 4)), _cplx((2, 4, 4))
    assert lib().orc_floq2spins_operators(D1, D2, J, gamma, _dp(H), _dp(L), _dp(K)) == 0
    return H, L, K


def floqnspins_operators(n, Delta, J, gamma):
    """FloqManySpins (sys_id 8): H (= special), L [n], K = hamiltonians_qj[0] (d = 2^n)."""
    d = 1 << n
    H, K, L = _cplx((d, d)), _cplx((d, d)), _cplx((n, d, d))
    assert lib().orc_floqnspins_operators(n, Delta, J, gamma, _dp(H), _dp(L), _dp(K)) == 0
    return H, L, K


def floqspph_operators(n_ph, Delta, Omega, gamma):
    """FloqSpinPh (sys_id 9): H (= special), L [1], K = hamiltonians_qj[0] (d = 2 (n_ph + 1))."""
    d = 2 * (n_ph + 1)
    H, K, L = _cplx((d, d)), _cplx((d, d)), _cplx((1, d, d))
    assert lib().orc_floqspph_operators(n_ph, Delta, Omega, gamma, _dp(H), _dp(L), _dp(K)) == 0
    return H, L, K


def integrable_operators(N, seed, num_seeds, tau, k):
    """Integrable (sys_id 5): L [N], special, K = hamiltonians_qj[0] (d = 2^N, H = 0)."""
    d = 1 << N
    L, S, K = _cplx((N, d, d)), _cplx((d, d)), _cplx((d, d))
    assert lib().orc_integrable_operators(N, seed, num_seeds, tau, k, _dp(L), _dp(S), _dp(K)) == 0
    return L, S, K


def mbl_imbalance(Nc, adr):
    """get_imbalance_mbl of each row of adr [n][d]."""
    adr = np.ascontiguousarray(adr, dtype=np.float64)
    out = np.zeros(adr.shape[0])
    lib().orc_mbl_imbalance(Nc, adr.shape[1], adr.shape[0], _dp(adr), _dp(out))
    return out


def dimer_heff(N, J, U, E, g):
    """H_eff = H - (i/2) (g/N) L^H L of the dimer (the RK propagator's non-drive part)."""
    out = _cplx((N + 1, N + 1))
    assert lib().orc_dimer_heff(N, J, U, E, g, _dp(out)) == 0
    return out


def expm(A):
    A = np.ascontiguousarray(A, dtype=np.complex128)
    out = np.empty_like(A)
    assert lib().orc_expm(A.shape[0], _dp(A), _dp(out)) == 0
    return out


def split_tree(K, T, deep):
    K = np.ascontiguousarray(K, dtype=np.complex128)
    d = K.shape[0]
    out = np.empty((deep, d, d), dtype=np.complex128)
    assert lib().orc_split_tree(d, _dp(K), T, deep, _dp(out)) == 0
    return out


def philox4x32_10(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return list(o)


def philox_uniform(seed, tr, idx):
    return lib().orc_philox_uniform(seed, tr, idx)


def matvec(M, x):
    M = np.ascontiguousarray(M, dtype=np.complex128)
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    lib().orc_matvec(M.shape[0], _dp(M), _dp(x), _dp(out))
    return out


def norm_square(x):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    return lib().orc_norm_square(x.shape[0], _dp(x))


def purity(psi):
    """Ensemble purity of states psi [n][d] and the trajectory-averaged rho (orc_purity)."""
    psi = np.ascontiguousarray(psi, dtype=np.complex128)
    n, d = psi.shape
    rho = np.zeros((d, d), np.complex128)
    return lib().orc_purity(d, n, _dp(psi), _dp(rho)), rho


def dump_periods(dump_type, dump_num, num_obs_periods):
    out = np.zeros(dump_num + 2, dtype=np.int32)
    n = lib().orc_dump_periods(dump_type, dump_num, num_obs_periods, out.ctypes.data_as(c_int_p))
    assert n > 0
    return out[:n].copy()


class Ensemble:
    """One QJ ensemble run by the oracle, mirroring the Std task flow."""

    def __init__(self, U, L, g, HE, R, T, n_traj, seed=0, record=2, rng_kind=0, inj_u=None, inj_off=None,
                 rec_cap=4096, tr_base=0, branch_len=None):
        self.U = np.ascontiguousarray(U, dtype=np.complex128)  # [nb, deep, d, d]
        nb, deep, d, _ = self.U.shape
        self.L = np.ascontiguousarray(L, dtype=np.complex128).reshape(-1, d, d)
        self.g = np.ascontiguousarray(g, dtype=np.float64)
        self.HE = np.ascontiguousarray(HE, dtype=np.complex128)
        self.R = np.ascontiguousarray(R if R is not None and len(R) else np.zeros((0, d, d)), dtype=np.complex128)
        self.d, self.n, self.deep, self.nb = d, n_traj, deep, nb
        self.inj_u = None if inj_u is None else np.ascontiguousarray(inj_u, dtype=np.float64)
        self.inj_off = None if inj_off is None else np.ascontiguousarray(inj_off, dtype=np.int64)
        p = OrcProblem()
        p.d, p.n_traj, p.deep, p.num_branches = d, n_traj, deep, nb
        p.num_diss, p.num_robs, p.record, p.rng_kind = self.L.shape[0], self.R.shape[0], record, rng_kind
        p.T, p.seed, p.tr_base = T, seed, tr_base
        p.U, p.L, p.g, p.HE = _dp(self.U), _dp(self.L), _dp(self.g), _dp(self.HE)
        p.R = _dp(self.R) if self.R.size else None
        p.inj_u = _dp(self.inj_u)
        p.inj_off = self.inj_off.ctypes.data_as(c_i64_p) if self.inj_off is not None else None
        self.branch_len = None if branch_len is None else np.ascontiguousarray(branch_len, np.float64)
        p.branch_len = _dp(self.branch_len)
        self.p = p
        n = n_traj
        self.phi = _cplx((n, d))
        self.eta = np.zeros(n)
        self.t = np.zeros(n)
        self.rng_pos = np.zeros(n, np.int64)
        self.jumps_counts = np.zeros(n, np.int32)
        self.matvecs = np.zeros(n, np.int64)
        self.rec_cap = rec_cap
        self.n_rec = np.zeros(n, np.int32)
        self.jump_times = np.zeros((n, rec_cap))
        self.jump_norms = np.zeros((n, rec_cap))
        self.jump_etas = np.zeros((n, rec_cap))
        self.diss_types = np.zeros((n, rec_cap), np.int32)
        self.error = np.zeros(n, np.int32)
        s = OrcState()
        s.phi, s.eta, s.t = _dp(self.phi), _dp(self.eta), _dp(self.t)
        s.rng_pos = self.rng_pos.ctypes.data_as(c_i64_p)
        s.jumps_counts = self.jumps_counts.ctypes.data_as(c_int_p)
        s.matvecs = self.matvecs.ctypes.data_as(c_i64_p)
        s.rec_cap = rec_cap
        s.n_rec = self.n_rec.ctypes.data_as(c_int_p)
        s.jump_times, s.jump_norms, s.jump_etas = _dp(self.jump_times), _dp(self.jump_norms), _dp(self.jump_etas)
        s.diss_types = self.diss_types.ctypes.data_as(c_int_p)
        s.error = self.error.ctypes.data_as(c_int_p)
        self.rng_src = np.arange(n, dtype=np.int32)
        s.rng_src = self.rng_src.ctypes.data_as(c_int_p)
        self.s = s
        self.mean_start = np.zeros(n)

    def init(self, start_type=0, start_state=0):
        lib().orc_init(C.byref(self.p), C.byref(self.s), start_type, start_state)

    def run_periods(self, n_periods, is_obs=1, tr0=0, tr1=None, n_threads=0):
        tr1 = self.n if tr1 is None else tr1
        return lib().orc_run_periods(C.byref(self.p), C.byref(self.s), tr0, tr1, n_periods, is_obs, n_threads)

    def run_branch_units(self, b, n_units, is_obs=1, tr0=0, tr1=None, n_threads=0):
        """n_units runs of branch b from level 0 (deep tasks: a sub-period is two units)."""
        tr1 = self.n if tr1 is None else tr1
        return lib().orc_run_branch_units(C.byref(self.p), C.byref(self.s), tr0, tr1, b, n_units, is_obs, n_threads)

    def run_periods_rk(self, n_periods, ND, DR, E0, A, rk_ns, period0=0, drv_type=0, freq=1.0, phase=0.0, is_obs=1,
                       tr0=0, tr1=None, n_threads=0):
        """RK propagator (prop_id 1) for n_periods periods numbered from period0."""
        tr1 = self.n if tr1 is None else tr1
        self._nd = np.ascontiguousarray(ND, dtype=np.complex128)
        self._dr = np.ascontiguousarray(DR, dtype=np.complex128)
        rk = OrcRk()
        rk.ND, rk.DR = _dp(self._nd), _dp(self._dr)
        rk.E0, rk.A, rk.freq, rk.phase, rk.drv_type, rk.rk_ns = E0, A, freq, phase, drv_type, rk_ns
        return lib().orc_run_periods_rk(C.byref(self.p), C.byref(rk), C.byref(self.s), tr0, tr1, n_periods, period0,
                                        is_obs, n_threads)

    def observables(self, is_start=False, want_adr=False):
        n, d = self.n, self.d
        out = {k: np.zeros(n) for k in ("norm", "mean", "dispersion", "m2", "energy")}
        robs = np.zeros((n, max(self.R.shape[0], 1)), np.complex128)
        adr = np.zeros((n, d)) if want_adr else None
        lib().orc_observables(C.byref(self.p), C.byref(self.s), int(is_start), _dp(self.mean_start),
                              _dp(out["norm"]), _dp(out["mean"]), _dp(out["dispersion"]), _dp(out["m2"]),
                              _dp(out["energy"]), _dp(robs), _dp(adr))
        out["random_obs"] = robs[:, : self.R.shape[0]]
        if want_adr:
            out["adr"] = adr
        return out

    def jumps(self, tr):
        k = int(self.n_rec[tr])
        return (self.jump_times[tr, :k].copy(), self.diss_types[tr, :k].copy(),
                self.jump_norms[tr, :k].copy(), self.jump_etas[tr, :k].copy())


class Lpn:
    """Lyapunov paired trajectories (task_id 7, LpnMult) over an Ensemble: bases [0, n/2),
    variation n/2 + b of base b (orc_lpn_start / orc_lpn_period in lpn_oracle.c)."""

    def __init__(self, ens, lpn_type=-1, eps_deep=100, eps_low=-10.0, eps_high=10.0, eps_error=1e-10,
                 delta_s=1e-3, delta_f_high=1e-1, delta_f_low=1e-5, per_period=0, max_energy=1.0, mbl_Nc=0,
                 spec_div=1.0, chars_sys=None):
        self.ens = ens
        n = ens.n
        self.cfg = OrcLpnConfig(lpn_type=lpn_type, eps_deep=eps_deep, per_period=int(per_period), eps_low=eps_low,
                                eps_high=eps_high, eps_error=eps_error, delta_s=delta_s,
                                delta_f_high=delta_f_high, delta_f_low=delta_f_low, max_energy=max_energy,
                                mbl_Nc=mbl_Nc, spec_div=spec_div,
                                chars_sys=(3 if mbl_Nc else 0) if chars_sys is None else chars_sys)
        self.a = {k: np.zeros(n) for k in ("lambda", "lambda_now", "delta_s", "mean_lpn", "energy_lpn", "ratio",
                                           "ds_rec", "df_rec", "eps")}
        self.robs_lpn = np.zeros((n, max(ens.R.shape[0], 1)), np.complex128)
        self.num_renorms = np.zeros(n, np.int32)
        self.renormed = np.zeros(n, np.int32)
        self.eps_iters = np.zeros(n, np.int32)
        self.var_pos = np.zeros(n, np.int64)
        s = OrcLpn()
        s.lambda_, s.lambda_now, s.delta_s = _dp(self.a["lambda"]), _dp(self.a["lambda_now"]), _dp(self.a["delta_s"])
        s.mean_lpn, s.energy_lpn = _dp(self.a["mean_lpn"]), _dp(self.a["energy_lpn"])
        s.robs_lpn = _dp(self.robs_lpn)
        s.num_renorms, s.renormed = self.num_renorms.ctypes.data_as(c_int_p), self.renormed.ctypes.data_as(c_int_p)
        s.var_pos = self.var_pos.ctypes.data_as(c_i64_p)
        s.ratio, s.ds_rec, s.df_rec, s.eps = _dp(self.a["ratio"]), _dp(self.a["ds_rec"]), _dp(self.a["df_rec"]), \
            _dp(self.a["eps"])
        s.eps_iters = self.eps_iters.ctypes.data_as(c_int_p)
        self.s = s

    def start(self):
        st = lib().orc_lpn_start(C.byref(self.ens.p), C.byref(self.ens.s), C.byref(self.cfg), C.byref(self.s))
        assert st == 0, st

    def period(self, curr_time):
        st = lib().orc_lpn_period(C.byref(self.ens.p), C.byref(self.ens.s), C.byref(self.cfg), C.byref(self.s),
                                  float(curr_time))
        assert st == 0, st

    def bases(self):
        st = lib().orc_lpn_bases(C.byref(self.ens.p), C.byref(self.ens.s), C.byref(self.cfg), C.byref(self.s))
        assert st == 0, st

    def values(self):
        out = {k: self.a[k].copy() for k in ("lambda_now", "lambda", "delta_s", "mean_lpn", "energy_lpn")}
        out["robs_lpn"] = self.robs_lpn[:, : self.ens.R.shape[0]].copy()
        out["num_renorms"] = self.num_renorms.copy()
        return out

    def last(self):
        return {"renormed": self.renormed.copy(), "ratio": self.a["ratio"].copy(), "delta_s": self.a["ds_rec"].copy(),
                "delta_f": self.a["df_rec"].copy(), "eps_iters": self.eps_iters.copy(), "eps": self.a["eps"].copy()}


def lpn_exp10(x):
    return lib().orc_lpn_exp10(float(x))


def lpn_log(x):
    return lib().orc_lpn_log(float(x))


# ---------------------------------------------------------------- f-basis
def _fb_sigs(L):
    if getattr(L, "_fb_ready", False):
        return
    ip = C.POINTER(C.c_int)
    L.orc_fb_operators.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double] + [c_double_p] * 3
    L.orc_fb_dense.argtypes = [C.c_int] + [C.c_double] * 4 + [c_double_p] * 3
    L.orc_fb_rk4.argtypes = ([C.c_int, ip, ip, c_double_p, ip, ip, c_double_p, c_double_p, C.c_double, C.c_double,
                              C.c_double, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, c_double_p])
    L.orc_fb_rho.argtypes = [C.c_int, c_double_p, c_double_p]
    L.orc_fb_rho.restype = None
    L.orc_fb_x_from_rho.argtypes = [C.c_int, c_double_p, c_double_p]
    L.orc_fb_x_from_rho.restype = None
    L._fb_ready = True


def fb_operators(N, J, U, E):
    L = lib()
    _fb_sigs(L)
    d = N + 1
    Hb, Hd, Lm = _cplx((d, d)), _cplx((d, d)), _cplx((d, d))
    L.orc_fb_operators(N, J, U, E, _dp(Hb), _dp(Hd), _dp(Lm))
    return Hb, Hd, Lm


def fb_dense(N, J, U, E, g):
    """Dense Gs, Qs_drv (n x n) and Ks (n), n = (N+1)^2 - 1."""
    L = lib()
    _fb_sigs(L)
    n = (N + 1) ** 2 - 1
    Gs, Qs, Ks = np.zeros((n, n)), np.zeros((n, n)), np.zeros(n)
    assert L.orc_fb_dense(N, J, U, E, g, _dp(Gs), _dp(Qs), _dp(Ks)) == 0
    return Gs, Qs, Ks


def fb_csr(M, rel_tol=1e-14):
    """CSR (indptr, indices, data) of a dense f-basis matrix; entries below rel_tol * max|M| are
    structural zeros of the Liouvillian left by rounding in the projection."""
    import scipy.sparse as sp

    A = np.where(np.abs(M) > rel_tol * np.abs(M).max(), M, 0.0)
    S = sp.csr_matrix(A)
    S.sort_indices()
    return S


def fb_rk4(Gs, Qs, Ks, x, A, freq=1.0, phase=0.0, drv_type=0, T=2 * np.pi, num_steps=1000, period0=0, n_periods=1):
    L = lib()
    _fb_sigs(L)
    ip = C.POINTER(C.c_int)
    g = (np.ascontiguousarray(Gs.indptr, np.int32), np.ascontiguousarray(Gs.indices, np.int32),
         np.ascontiguousarray(Gs.data, np.float64))
    q = (np.ascontiguousarray(Qs.indptr, np.int32), np.ascontiguousarray(Qs.indices, np.int32),
         np.ascontiguousarray(Qs.data, np.float64))
    x = np.ascontiguousarray(x, np.float64).copy()
    Ks = np.ascontiguousarray(Ks, np.float64)
    assert L.orc_fb_rk4(len(x), g[0].ctypes.data_as(ip), g[1].ctypes.data_as(ip), _dp(g[2]), q[0].ctypes.data_as(ip),
                        q[1].ctypes.data_as(ip), _dp(q[2]), _dp(Ks), A, freq, phase, drv_type, T, num_steps,
                        period0, n_periods, _dp(x)) == 0
    return x


def fb_rho(N, x):
    L = lib()
    _fb_sigs(L)
    rho = _cplx((N + 1, N + 1))
    L.orc_fb_rho(N, _dp(np.ascontiguousarray(x, np.float64)), _dp(rho))
    return rho


def fb_x_from_rho(N, rho):
    L = lib()
    _fb_sigs(L)
    x = np.zeros((N + 1) ** 2 - 1)
    L.orc_fb_x_from_rho(N, _dp(np.ascontiguousarray(rho, np.complex128)), _dp(x))
    return x
