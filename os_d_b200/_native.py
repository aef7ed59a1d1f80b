"""ctypes binding of libqjx_b200.so (the C ABI in include/qjx_b200.h).

The library is the product: there is no Python or CPU fallback.  If the shared object
is missing or lacks a symbol, loading fails with an error.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqjx_b200.so")

c_double_p = C.POINTER(C.c_double)
c_int_p = C.POINTER(C.c_int)
c_i64_p = C.POINTER(C.c_int64)

# every entry point declared in include/qjx_b200.h
EXPORTS = [
    "qjx_create", "qjx_create_rk", "qjx_build_dimer_rk", "qjx_build_dimer_deep", "qjx_destroy", "qjx_last_error", "qjx_status_string", "qjx_set_states", "qjx_set_uniforms",
    "qjx_init_thresholds", "qjx_run_periods", "qjx_reset_times", "qjx_observe", "qjx_get_observables",
    "qjx_get_mean_start", "qjx_purity", "qjx_get_states", "qjx_jump_count", "qjx_get_jumps", "qjx_get_stats",
    "qjx_set_trace", "qjx_get_trace", "qjx_measure_fp64_peak", "qjx_autotune", "qjx_expm_tree", "qjx_mem_info", "qjx_engine_bytes", "qjx_build_dimer", "qjx_expm",
    "qjx_random_observables", "qjx_build_jcs", "qjx_mbl_size", "qjx_build_mbl", "qjx_mbl_imbalance", "qjx_build_integrable", "qjx_build_ps", "qjx_build_floq2spins", "qjx_build_floqnspins", "qjx_build_floqspph", "qjx_create_batch", "qjx_create_slots", "qjx_slot_load", "qjx_slot_release",
    "qjx_set_active", "qjx_set_bases_only", "qjx_checkpoint_size", "qjx_checkpoint_save", "qjx_checkpoint_load", "qjx_lpn_start", "qjx_lpn_period", "qjx_lpn_bases", "qjx_run_sub_periods", "qjx_lpn_get",
    "qjx_lpn_get_last", "qjx_fb_rk4_noalloc", "qjx_fb_build_dimer", "qjx_fb_create", "qjx_fb_run", "qjx_fb_info", "qjx_fb_get", "qjx_fb_destroy",
]


class QjxTiles(C.Structure):
    _fields_ = [("nc", C.c_int), ("kb", C.c_int), ("stages", C.c_int), ("rows", C.c_int)]


class QjxConfig(C.Structure):
    _fields_ = [("d", C.c_int), ("n_traj", C.c_int), ("deep", C.c_int), ("num_branches", C.c_int),
                ("num_diss", C.c_int), ("num_robs", C.c_int), ("T", C.c_double), ("record", C.c_int),
                ("rng_kind", C.c_int), ("seed", C.c_uint64), ("rec_cap", C.c_int), ("keep_adr", C.c_int),
                ("max_dumps", C.c_int), ("device", C.c_int), ("tr_base", C.c_int64), ("deep_num_steps", C.c_int),
                ("precision", C.c_int), ("branch_len", c_double_p), ("split_recheck", C.c_double),
                ("tiles", QjxTiles)]


class QjxEnsemble(C.Structure):
    _fields_ = [("d", C.c_int), ("n_traj", C.c_int), ("T", C.c_double), ("seed", C.c_uint64),
                ("tr_base", C.c_int64), ("U", c_double_p), ("L", c_double_p), ("g", c_double_p),
                ("HE", c_double_p), ("R", c_double_p)]


class QjxLpnConfig(C.Structure):
    _fields_ = [("lpn_type", C.c_int), ("eps_deep", C.c_int), ("per_period", C.c_int), ("pad", C.c_int),
                ("eps_low", C.c_double), ("eps_high", C.c_double), ("eps_error", C.c_double),
                ("delta_s", C.c_double), ("delta_f_high", C.c_double), ("delta_f_low", C.c_double),
                ("max_energy", C.c_double), ("mbl_Nc", C.c_int), ("chars_sys", C.c_int), ("spec_div", C.c_double)]


class QjxStats(C.Structure):
    _fields_ = [("micro_steps", C.c_int64), ("matvecs", C.c_int64), ("jumps", C.c_int64),
                ("kernel_ms", C.c_double), ("last_call_ms", C.c_double), ("step_kernel_ms", C.c_double),
                ("launches", C.c_int64), ("mma_tiles", C.c_int64), ("rechecks", C.c_int64)]


_lib = None


class QjxError(RuntimeError):
    pass


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise QjxError(f"native library missing: {LIB_PATH} (run os_d_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        for name in EXPORTS:
            if not hasattr(L, name):
                raise QjxError(f"native library lacks {name}")
        vp = C.c_void_p
        L.qjx_create.argtypes = [C.POINTER(QjxConfig)] + [c_double_p] * 5 + [C.POINTER(vp)]
        L.qjx_create_rk.argtypes = ([C.POINTER(QjxConfig), c_double_p, c_double_p, C.c_double, C.c_double, C.c_int,
                                     C.c_double, C.c_double, C.c_int] + [c_double_p] * 4 + [C.POINTER(vp)])
        L.qjx_destroy.argtypes = [vp]
        L.qjx_destroy.restype = None
        L.qjx_last_error.argtypes = [vp]
        L.qjx_last_error.restype = C.c_char_p
        L.qjx_status_string.argtypes = [C.c_int]
        L.qjx_status_string.restype = C.c_char_p
        L.qjx_set_states.argtypes = [vp, c_double_p]
        L.qjx_set_uniforms.argtypes = [vp, c_double_p, c_i64_p]
        L.qjx_init_thresholds.argtypes = [vp]
        L.qjx_run_periods.argtypes = [vp, C.c_int, C.c_int, c_int_p, C.c_int, C.c_int]
        L.qjx_reset_times.argtypes = [vp]
        L.qjx_observe.argtypes = [vp, C.c_int, C.c_int]
        L.qjx_get_observables.argtypes = [vp, C.c_int, C.c_int] + [c_double_p] * 7
        L.qjx_get_mean_start.argtypes = [vp, c_double_p]
        L.qjx_purity.argtypes = [vp, c_double_p, c_double_p]
        L.qjx_get_states.argtypes = [vp, c_double_p, c_double_p, c_double_p, c_int_p]
        L.qjx_jump_count.argtypes = [vp, C.c_int, c_i64_p]
        L.qjx_get_jumps.argtypes = [vp, C.c_int, c_double_p, c_int_p, c_double_p, c_double_p]
        L.qjx_get_stats.argtypes = [vp, C.POINTER(QjxStats)]
        L.qjx_set_trace.argtypes = [vp, C.c_int]
        L.qjx_set_active.argtypes = [vp, C.c_int]
        L.qjx_set_bases_only.argtypes = [vp, C.c_int]
        L.qjx_checkpoint_size.argtypes = [vp, C.POINTER(C.c_size_t)]
        L.qjx_checkpoint_save.argtypes = [vp, vp, C.c_size_t]
        L.qjx_checkpoint_load.argtypes = [vp, vp, C.c_size_t]
        L.qjx_create_batch.argtypes = [C.POINTER(QjxConfig), C.c_int, C.POINTER(QjxEnsemble), C.POINTER(vp)]
        L.qjx_create_slots.argtypes = [C.POINTER(QjxConfig), C.c_int, C.c_int, C.c_int, C.POINTER(vp)]
        L.qjx_slot_load.argtypes = [vp, C.c_int, C.POINTER(QjxEnsemble), c_double_p]
        L.qjx_slot_release.argtypes = [vp, C.c_int]
        L.qjx_lpn_start.argtypes = [vp, C.POINTER(QjxLpnConfig)]
        L.qjx_lpn_period.argtypes = [vp, C.c_double, C.c_int]
        L.qjx_lpn_bases.argtypes = [vp]
        L.qjx_run_sub_periods.argtypes = [vp, C.c_int, C.c_int]
        L.qjx_lpn_get.argtypes = [vp] + [c_double_p] * 6 + [c_int_p]
        L.qjx_lpn_get_last.argtypes = [vp, c_int_p, c_double_p, c_double_p, c_double_p, c_int_p, c_double_p]
        L.qjx_get_trace.argtypes = [vp, c_i64_p, c_int_p, c_int_p]
        L.qjx_measure_fp64_peak.argtypes = [C.c_int, c_double_p, c_double_p]
        L.qjx_autotune.argtypes = ([C.POINTER(QjxConfig)] + [c_double_p] * 4 +
                                   [C.c_int, C.POINTER(QjxTiles), C.POINTER(QjxTiles), c_double_p, c_int_p])
        L.qjx_build_dimer.argtypes = [C.c_int] + [C.c_double] * 6 + [C.c_int] + [c_double_p] * 5
        L.qjx_build_dimer_deep.argtypes = [C.c_int] + [C.c_double] * 6 + [C.c_int, C.c_int] + [c_double_p] * 5
        L.qjx_expm.argtypes = [C.c_int, c_double_p, c_double_p]
        L.qjx_expm_tree.argtypes = [C.c_int, C.c_int, c_double_p, c_double_p, C.c_int, C.c_int, c_double_p]
        L.qjx_mem_info.argtypes = [C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
        L.qjx_engine_bytes.argtypes = [vp, C.POINTER(C.c_size_t)]
        L.qjx_build_jcs.argtypes = [C.c_int] + [C.c_double] * 4 + [C.c_int] + [c_double_p] * 7
        L.qjx_mbl_size.argtypes = [C.c_int, C.c_int, c_int_p, c_int_p]
        L.qjx_build_mbl.argtypes = ([C.c_int] + [C.c_double] * 3 + [C.c_int] * 3 + [C.c_double] * 3 + [C.c_int]
                                    + [c_double_p, c_int_p] + [c_double_p] * 4)
        L.qjx_mbl_imbalance.argtypes = [C.c_int, C.c_int, c_double_p, c_double_p]
        L.qjx_build_ps.argtypes = ([C.c_int] * 2 + [C.c_double] * 4 + [C.c_int] + [C.c_double] * 3 + [C.c_int]
                                   + [c_double_p] * 6)
        L.qjx_build_floq2spins.argtypes = [C.c_double] * 5 + [C.c_int] + [c_double_p] * 4
        L.qjx_build_floqnspins.argtypes = [C.c_int] + [C.c_double] * 4 + [C.c_int] + [c_double_p] * 4
        L.qjx_build_floqspph.argtypes = [C.c_int] + [C.c_double] * 4 + [C.c_int] + [c_double_p] * 4
        L.qjx_build_integrable.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [C.c_int] + [c_double_p] * 4
        L.qjx_build_dimer_rk.argtypes = [C.c_int] + [C.c_double] * 4 + [c_double_p] * 2
        L.qjx_fb_build_dimer.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                         C.POINTER(C.c_int), C.POINTER(C.c_int), c_int_p, c_int_p, c_double_p,
                                         c_int_p, c_int_p, c_double_p, c_double_p]
        L.qjx_random_observables.argtypes = [C.c_int] * 5 + [c_double_p]
        L.qjx_fb_create.argtypes = ([C.c_int, c_int_p, c_int_p, c_double_p, c_int_p, c_int_p, c_double_p,
                                     c_double_p, c_double_p, C.c_double, C.c_double, C.c_double, C.c_int,
                                     C.c_double, C.c_int, C.c_int, C.POINTER(vp)])
        L.qjx_fb_run.argtypes = [vp, C.c_int, C.c_int]
        L.qjx_fb_get.argtypes = [vp, c_double_p, c_double_p]
        L.qjx_fb_info.argtypes = [vp, c_int_p]
        L.qjx_fb_rk4_noalloc.argtypes = ([C.c_int] + [vp] * 8 + [C.c_double] * 3 + [C.c_int, C.c_double]
                                         + [C.c_int] * 4 + [vp])
        L.qjx_fb_destroy.argtypes = [vp]
        L.qjx_fb_destroy.restype = None
        _lib = L
    return _lib


def dp(a):
    return None if a is None else a.ctypes.data_as(c_double_p)


def ip(a):
    return None if a is None else a.ctypes.data_as(c_int_p)


def check(status, handle=None, what=""):
    if status != 0:
        msg = lib().qjx_status_string(status).decode()
        detail = lib().qjx_last_error(handle).decode() if handle else lib().qjx_last_error(None).decode()
        if detail:
            msg += ": " + detail
        raise QjxError(f"{what} failed ({status}): {msg}")


def build_dimer(N, J, U, E, A, g, omega, deep):
    """Dimer operators and split propagators built by the library (host FP64)."""
    d = N + 1
    H = np.zeros((d, d), np.complex128)
    Hd = np.zeros_like(H)
    Lm = np.zeros_like(H)
    Ut = np.zeros((2, deep, d, d), np.complex128)
    check(lib().qjx_build_dimer(N, J, U, E, A, g, omega, deep, dp(H), dp(Hd), dp(Lm), None, dp(Ut)),
          what="qjx_build_dimer")
    return H, Hd, Lm, Ut


def build_dimer_deep(N, J, U, E, A, g, omega, deep, deep_num_steps):
    """build_dimer with the split tree of the deep tasks' sub-period T / (2 deep_num_steps)."""
    d = N + 1
    H = np.zeros((d, d), np.complex128)
    Hd = np.zeros_like(H)
    Lm = np.zeros_like(H)
    Ut = np.zeros((2, deep, d, d), np.complex128)
    check(lib().qjx_build_dimer_deep(N, J, U, E, A, g, omega, deep, deep_num_steps, dp(H), dp(Hd), dp(Lm), None,
                                     dp(Ut)), what="qjx_build_dimer_deep")
    return H, Hd, Lm, Ut


def build_jcs(N, alpha, drv_ampl, part_1, part_2, deep):
    """JCS system (sys_id 1): H, H_drv, L = a, Nop = a^+ a, A = a and the split trees [2][deep][N][N];
    a period runs part b (head part_b * alpha) as two halves: engine branches [U0, U0, U1, U1] with
    branch_len [h0, h0, h1, h1] / 2."""
    d = N
    H, Hd, L, Nop, A = (np.zeros((d, d), np.complex128) for _ in range(5))
    U = np.zeros((2, deep, d, d), np.complex128)
    check(lib().qjx_build_jcs(N, alpha, drv_ampl, part_1, part_2, deep, dp(H), dp(Hd), dp(L), dp(Nop), dp(A), None,
                              dp(U)), what="qjx_build_jcs")
    return H, Hd, L, Nop, A, U


def build_mbl(Nc, W, U, J, mbl_seed, mbl_mns, diss_type, diss_phase, gamma, T, deep):
    """MBL system (sys_id 3): energies [Nc], basis words [d], H, L [num_diss] and the split tree
    [deep][d][d] of one branch (a period runs it twice); jump rates are 1."""
    d, nd = C.c_int(), C.c_int()
    check(lib().qjx_mbl_size(Nc, diss_type, C.byref(d), C.byref(nd)), what="qjx_mbl_size")
    d, nd = d.value, nd.value
    en = np.zeros(Nc)
    xs = np.zeros(d, np.int32)
    H = np.zeros((d, d), np.complex128)
    Lm = np.zeros((nd, d, d), np.complex128)
    Ut = np.zeros((deep, d, d), np.complex128)
    check(lib().qjx_build_mbl(Nc, W, U, J, mbl_seed, mbl_mns, diss_type, diss_phase, gamma, T, deep, dp(en),
                              xs.ctypes.data_as(c_int_p), dp(H), dp(Lm), None, dp(Ut)), what="qjx_build_mbl")
    return en, xs, H, Lm, Ut


def build_ps(ns, nps, alpha, d_prm, g_prm, drv_ampl, diss_type, diss_w, part_1, part_2, deep):
    """PS system (sys_id 2): H, Hd, L [1 + ns diss_type], S [4] (spec, spec_2, spec_3, photons) and the
    split trees [2][deep][d][d] (part b's head part_b alpha, run as two halves)."""
    d = (1 << ns) * nps
    nd = 1 if diss_type == 0 else 1 + ns
    H, Hd = np.zeros((d, d), np.complex128), np.zeros((d, d), np.complex128)
    Lm, S = np.zeros((nd, d, d), np.complex128), np.zeros((4, d, d), np.complex128)
    Ut = np.zeros((2, deep, d, d), np.complex128)
    check(lib().qjx_build_ps(ns, nps, alpha, d_prm, g_prm, drv_ampl, diss_type, diss_w, part_1, part_2, deep, dp(H),
                             dp(Hd), dp(Lm), dp(S), None, dp(Ut)), what="qjx_build_ps")
    return H, Hd, Lm, S, Ut


def build_floq2spins(D1, D2, J, gamma, T, deep):
    """Floquet two-spin system (sys_id 7), QJ branch: H (= special), L [2], split tree [deep][4][4]."""
    H, Lm, Ut = np.zeros((4, 4), np.complex128), np.zeros((2, 4, 4), np.complex128), np.zeros((deep, 4, 4), np.complex128)
    check(lib().qjx_build_floq2spins(D1, D2, J, gamma, T, deep, dp(H), dp(Lm), None, dp(Ut)), what="qjx_build_floq2spins")
    return H, Lm, Ut


def build_floqnspins(n, Delta, J, gamma, T, deep):
    """Floquet many-spin system (sys_id 8), QJ branch: H (= special), L [n], split tree [deep][d][d]."""
    d = 1 << n
    H, Lm, Ut = (np.zeros((d, d), np.complex128), np.zeros((n, d, d), np.complex128),
                 np.zeros((deep, d, d), np.complex128))
    check(lib().qjx_build_floqnspins(n, Delta, J, gamma, T, deep, dp(H), dp(Lm), None, dp(Ut)),
          what="qjx_build_floqnspins")
    return H, Lm, Ut


def build_floqspph(n_ph, Delta, Omega, gamma, T, deep):
    """Floquet spin-photon system (sys_id 9), QJ branch: H (= special), L [1], split tree [deep][d][d]."""
    d = 2 * (n_ph + 1)
    H, Lm, Ut = (np.zeros((d, d), np.complex128), np.zeros((1, d, d), np.complex128),
                 np.zeros((deep, d, d), np.complex128))
    check(lib().qjx_build_floqspph(n_ph, Delta, Omega, gamma, T, deep, dp(H), dp(Lm), None, dp(Ut)),
          what="qjx_build_floqspph")
    return H, Lm, Ut


def build_integrable(N, seed, num_seeds, tau, k, T, deep):
    """Integrable system (sys_id 5): L [N], the special (spec) matrix and the split tree [deep][d][d]
    of one branch (a period runs it twice); d = 2^N, H = 0, jump rates 1."""
    d = 1 << N
    Lm = np.zeros((N, d, d), np.complex128)
    S = np.zeros((d, d), np.complex128)
    Ut = np.zeros((deep, d, d), np.complex128)
    check(lib().qjx_build_integrable(N, seed, num_seeds, tau, k, T, deep, dp(Lm), dp(S), None, dp(Ut)),
          what="qjx_build_integrable")
    return Lm, S, Ut


def mbl_imbalance(Nc, adr):
    """The MBL imbalance of each probability row adr [n][d]."""
    adr = np.ascontiguousarray(adr, dtype=np.float64)
    out = np.zeros(adr.shape[0])
    check(lib().qjx_mbl_imbalance(Nc, adr.shape[0], dp(adr), dp(out)), what="qjx_mbl_imbalance")
    return out


def build_dimer_rk(N, J, U, E, g):
    """Operators of the RK propagator: H_eff = H - (i/2)(g/N) L^H L and H_drv."""
    d = N + 1
    He = np.zeros((d, d), np.complex128)
    Hd = np.zeros_like(He)
    check(lib().qjx_build_dimer_rk(N, J, U, E, g, dp(He), dp(Hd)), what="qjx_build_dimer_rk")
    return He, Hd


def dimer_generators(N, J, U, E, A, g):
    """The two non-Hermitian generators K_b = -i H_eff,b of the split propagators."""
    d = N + 1
    K = np.zeros((2, d, d), np.complex128)
    check(lib().qjx_build_dimer(N, J, U, E, A, g, 1.0, 1, None, None, None, dp(K), None), what="qjx_build_dimer")
    return K


def measure_fp64_peak(device=0):
    """(FFMA TFLOP/s, FP64 tensor-core DMMA TFLOP/s) measured on the device."""
    f, m = C.c_double(), C.c_double()
    check(lib().qjx_measure_fp64_peak(device, C.byref(f), C.byref(m)), what="qjx_measure_fp64_peak")
    return f.value, m.value


def random_observables(d, num, seed, mns, rtype):
    out = np.zeros((num, d, d), np.complex128)
    check(lib().qjx_random_observables(d, num, seed, mns, rtype, dp(out)), what="qjx_random_observables")
    return out


def fb_build_dimer(N, J, U, E, g):
    """f-basis Liouvillian of the dimer: (Gs, Qs) as (indptr, indices, data) CSR triples and Ks."""
    L = lib()
    gn, qn = C.c_int(0), C.c_int(0)
    check(L.qjx_fb_build_dimer(N, J, U, E, g, C.byref(gn), C.byref(qn), None, None, None, None, None, None, None),
          what="qjx_fb_build_dimer")
    n = (N + 1) ** 2 - 1
    gr, gc, gv = np.zeros(n + 1, np.int32), np.zeros(gn.value, np.int32), np.zeros(gn.value)
    qr, qc, qv = np.zeros(n + 1, np.int32), np.zeros(qn.value, np.int32), np.zeros(qn.value)
    ks = np.zeros(n)
    check(L.qjx_fb_build_dimer(N, J, U, E, g, C.byref(gn), C.byref(qn), ip(gr), ip(gc), dp(gv), ip(qr), ip(qc),
                               dp(qv), dp(ks)), what="qjx_fb_build_dimer")
    return (gr, gc, gv), (qr, qc, qv), ks


def build_dimer_gpu(N, J, U, E, A, g, omega, deep, device=0):
    """The dimer's H, Hd, L on the host and its split tree on the GPU (qjx_expm_tree): the outputs
    of build_dimer, the tree within about 1e-12 of the host's level-by-level exponentials."""
    d = N + 1
    H, Hd, L = (np.zeros((d, d), np.complex128) for _ in range(3))
    K = np.zeros((2, d, d), np.complex128)
    check(lib().qjx_build_dimer(N, J, U, E, A, g, omega, deep, dp(H), dp(Hd), dp(L), dp(K), None),
          what="qjx_build_dimer")
    T = 2.0 * 3.1415926535897932384626433832795 / omega
    Ut = np.zeros((2, deep, d, d), np.complex128)
    head = np.array([T, T])
    check(lib().qjx_expm_tree(d, 2, dp(K), dp(head), deep, device, dp(Ut)), what="qjx_expm_tree")
    return H, Hd, L, Ut


def mem_info(device=0):
    """(free, total) device bytes (cudaMemGetInfo)."""
    f, t = C.c_size_t(), C.c_size_t()
    check(lib().qjx_mem_info(device, C.byref(f), C.byref(t)), what="qjx_mem_info")
    return f.value, t.value


def expm(A):
    A = np.ascontiguousarray(A, np.complex128)
    out = np.empty_like(A)
    check(lib().qjx_expm(A.shape[0], dp(A), dp(out)), what="qjx_expm")
    return out
