"""Python handles over the C ABI (include/qjx_b200.h): QJ ensemble engine and f-basis RK4.

These mirror the reference's in-process strategy API for the Std task with the QJ
propagator (source/cpp/QJX/QJX/experiment.cpp:411-542: trans_process then obser_process),
batched over every trajectory of the ensemble.
"""
import ctypes as C

import numpy as np

from . import _native as N


class Engine:
    """One ensemble of trajectories resident on a GPU."""

    def __init__(self, U, L, g, HE, R=None, T=2 * np.pi, n_traj=1, seed=0, record=0, rng_kind=0, rec_cap=1024,
                 keep_adr=0, max_dumps=1, device=0, tr_base=0, precision=0, deep_num_steps=0, branch_len=None,
                 split_recheck=0.0, tiles=None):
        U = np.ascontiguousarray(U, np.complex128)
        nb, deep, d, _ = U.shape
        L = np.ascontiguousarray(L, np.complex128).reshape(-1, d, d)
        g = np.ascontiguousarray(np.atleast_1d(g), np.float64)
        HE = np.ascontiguousarray(HE, np.complex128)
        R = np.zeros((0, d, d), np.complex128) if R is None else np.ascontiguousarray(R, np.complex128).reshape(-1, d, d)
        cfg = N.QjxConfig()
        cfg.d, cfg.n_traj, cfg.deep, cfg.num_branches = d, n_traj, deep, nb
        cfg.num_diss, cfg.num_robs, cfg.T, cfg.record = L.shape[0], R.shape[0], T, record
        cfg.rng_kind, cfg.seed, cfg.rec_cap, cfg.keep_adr = rng_kind, seed, rec_cap, keep_adr
        cfg.max_dumps, cfg.device, cfg.tr_base = max_dumps, device, tr_base
        cfg.precision = precision  # 0 complex FP64, 1 split bf16x3 on tcgen05
        cfg.split_recheck = split_recheck  # split form: FP64 recheck band (0: default 1e-5, < 0: off)
        if tiles:  # explicit tile shapes (dict nc / kb / stages / rows); default: rule or autotuner cache
            cfg.tiles = N.QjxTiles(**tiles)
        cfg.deep_num_steps = deep_num_steps  # > 0: StdDeep task (U from build_dimer_deep)
        self._branch_len = None if branch_len is None else np.ascontiguousarray(branch_len, np.float64)
        cfg.branch_len = N.dp(self._branch_len)  # per-branch durations (None: T / 2 each)
        self.cfg = cfg
        self.d, self.n, self.nr = d, n_traj, R.shape[0]
        self.keep_adr = keep_adr
        h = C.c_void_p()
        N.check(N.lib().qjx_create(C.byref(cfg), N.dp(U), N.dp(L), N.dp(g), N.dp(HE), N.dp(R) if R.size else None,
                                   C.byref(h)), what="qjx_create")
        self.h = h

    @classmethod
    def rk(cls, H_eff, H_drv, L, g, HE, R=None, T=2 * np.pi, n_traj=1, E0=1.0, A=0.0, rk_ns=1000, drv_type=0,
           drv_freq=1.0, drv_phase=0.0, seed=0, record=0, rng_kind=0, rec_cap=1024, keep_adr=0, max_dumps=1,
           device=0, tr_base=0):
        """Engine with the RK propagator (prop_id 1): RK4 of -i (H_eff + E(t) H_drv) with rk_ns steps
        per period and linear interpolation of the jump time."""
        H_eff = np.ascontiguousarray(H_eff, np.complex128)
        d = H_eff.shape[0]
        H_drv = np.ascontiguousarray(H_drv, np.complex128)
        self = cls.__new__(cls)
        L = np.ascontiguousarray(L, np.complex128).reshape(-1, d, d)
        g = np.ascontiguousarray(np.atleast_1d(g), np.float64)
        HE = np.ascontiguousarray(HE, np.complex128)
        R = np.zeros((0, d, d), np.complex128) if R is None else np.ascontiguousarray(R, np.complex128).reshape(-1, d, d)
        cfg = N.QjxConfig()
        cfg.d, cfg.n_traj, cfg.deep, cfg.num_branches = d, n_traj, 2, 1
        cfg.num_diss, cfg.num_robs, cfg.T, cfg.record = L.shape[0], R.shape[0], T, record
        cfg.rng_kind, cfg.seed, cfg.rec_cap, cfg.keep_adr = rng_kind, seed, rec_cap, keep_adr
        cfg.max_dumps, cfg.device, cfg.tr_base, cfg.precision = max_dumps, device, tr_base, 0
        self.cfg = cfg
        self.d, self.n, self.nr = d, n_traj, R.shape[0]
        self.keep_adr = keep_adr
        h = C.c_void_p()
        N.check(N.lib().qjx_create_rk(C.byref(cfg), N.dp(H_eff), N.dp(H_drv), E0, A, drv_type, drv_freq, drv_phase,
                                      rk_ns, N.dp(L), N.dp(g), N.dp(HE), N.dp(R) if R.size else None, C.byref(h)),
                what="qjx_create_rk")
        self.h = h
        return self

    @classmethod
    def batch(cls, ensembles, deep=16, num_branches=2, record=0, rng_kind=0, rec_cap=1024, keep_adr=0, max_dumps=1,
              device=0, deep_num_steps=0, precision=0, split_recheck=0.0):
        """Batched engine over ensembles of uneven dimension: each item is a dict with U
        ([nb][deep][d][d]), L, g, HE, optional R, n_traj, T, seed, tr_base.  Trajectories are numbered
        ensemble after ensemble (`ranges` gives each ensemble's slice); state rows have the largest d."""
        self = cls.__new__(cls)
        keep, arr = [], (N.QjxEnsemble * len(ensembles))()
        nr = None
        for i, e in enumerate(ensembles):
            U = np.ascontiguousarray(e["U"], np.complex128)
            d = U.shape[-1]
            L = np.ascontiguousarray(e["L"], np.complex128).reshape(-1, d, d)
            g = np.ascontiguousarray(np.atleast_1d(e.get("g", [1.0])), np.float64)
            HE = np.ascontiguousarray(e["HE"], np.complex128)
            R = e.get("R")
            R = np.zeros((0, d, d), np.complex128) if R is None else np.ascontiguousarray(R, np.complex128).reshape(-1, d, d)
            nr = R.shape[0] if nr is None else nr
            keep += [U, L, g, HE, R]
            arr[i] = N.QjxEnsemble(d=d, n_traj=int(e["n_traj"]), T=float(e.get("T", 2 * np.pi)),
                                   seed=int(e.get("seed", 0)), tr_base=int(e.get("tr_base", 0)), U=N.dp(U), L=N.dp(L),
                                   g=N.dp(g), HE=N.dp(HE), R=N.dp(R) if R.size else None)
        cfg = N.QjxConfig()
        cfg.deep, cfg.num_branches, cfg.num_diss, cfg.num_robs = deep, num_branches, keep[1].shape[0], nr
        cfg.record, cfg.rng_kind, cfg.rec_cap, cfg.keep_adr = record, rng_kind, rec_cap, keep_adr
        cfg.max_dumps, cfg.device, cfg.deep_num_steps, cfg.precision = max_dumps, device, deep_num_steps, precision
        cfg.split_recheck = split_recheck
        h = C.c_void_p()
        N.check(N.lib().qjx_create_batch(C.byref(cfg), len(ensembles), arr, C.byref(h)), what="qjx_create_batch")
        self.h = h
        self.cfg = cfg
        dims = [a.d for a in arr]
        self.d, self.n, self.nr = max(dims), sum(a.n_traj for a in arr), nr
        self.keep_adr = keep_adr
        starts = np.cumsum([0] + [a.n_traj for a in arr])
        self.ranges = [slice(int(starts[i]), int(starts[i + 1])) for i in range(len(arr))]
        self.dims = dims
        return self

    @staticmethod
    def _ensemble_struct(e, keep):
        U = np.ascontiguousarray(e["U"], np.complex128)
        d = U.shape[-1]
        L = np.ascontiguousarray(e["L"], np.complex128).reshape(-1, d, d)
        g = np.ascontiguousarray(np.atleast_1d(e.get("g", [1.0])), np.float64)
        HE = np.ascontiguousarray(e["HE"], np.complex128)
        R = e.get("R")
        R = np.zeros((0, d, d), np.complex128) if R is None else np.ascontiguousarray(R, np.complex128).reshape(-1, d, d)
        keep += [U, L, g, HE, R]
        return N.QjxEnsemble(d=d, n_traj=int(e["n_traj"]), T=float(e.get("T", 2 * np.pi)), seed=int(e.get("seed", 0)),
                             tr_base=int(e.get("tr_base", 0)), U=N.dp(U), L=N.dp(L), g=N.dp(g), HE=N.dp(HE),
                             R=N.dp(R) if R.size else None)

    @classmethod
    def slots(cls, n_slots, d_cap, n_cap, deep=16, num_branches=2, num_diss=1, num_robs=0, record=0, rng_kind=0,
              rec_cap=1024, keep_adr=0, max_dumps=1, device=0):
        """Serving engine: n_slots resident ensemble slots (dimension <= d_cap, n_cap trajectories
        each; slot s owns trajectories s * n_cap ...), loaded and released between run calls."""
        self = cls.__new__(cls)
        cfg = N.QjxConfig()
        cfg.deep, cfg.num_branches, cfg.num_diss, cfg.num_robs = deep, num_branches, num_diss, num_robs
        cfg.record, cfg.rng_kind, cfg.rec_cap, cfg.keep_adr = record, rng_kind, rec_cap, keep_adr
        cfg.max_dumps, cfg.device, cfg.precision = max_dumps, device, 0
        h = C.c_void_p()
        N.check(N.lib().qjx_create_slots(C.byref(cfg), n_slots, d_cap, n_cap, C.byref(h)), what="qjx_create_slots")
        self.h, self.cfg = h, cfg
        self.d, self.n, self.nr, self.keep_adr = d_cap, n_slots * n_cap, num_robs, keep_adr
        self.n_cap = n_cap
        return self

    def slot_load(self, slot, ensemble, psi=None):
        """Load an ensemble (dict as for Engine.batch) into a free slot; psi [n_traj][d] or None (|0>)."""
        keep = []
        st = self._ensemble_struct(ensemble, keep)
        p = None if psi is None else np.ascontiguousarray(psi, np.complex128)
        self._chk(N.lib().qjx_slot_load(self.h, slot, C.byref(st), N.dp(p)), "qjx_slot_load")

    def slot_release(self, slot):
        self._chk(N.lib().qjx_slot_release(self.h, slot), "qjx_slot_release")

    def _chk(self, st, what):
        N.check(st, self.h, what)

    def close(self):
        if self.h:
            N.lib().qjx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_states(self, psi):
        psi = np.ascontiguousarray(psi, np.complex128)
        assert psi.shape == (self.n, self.d)
        self._chk(N.lib().qjx_set_states(self.h, N.dp(psi)), "qjx_set_states")

    def set_uniforms(self, u, offsets):
        u = np.ascontiguousarray(u, np.float64)
        off = np.ascontiguousarray(offsets, np.int64)
        self._chk(N.lib().qjx_set_uniforms(self.h, N.dp(u), off.ctypes.data_as(N.c_i64_p)), "qjx_set_uniforms")

    def init_thresholds(self):
        self._chk(N.lib().qjx_init_thresholds(self.h), "qjx_init_thresholds")

    def run_periods(self, n_periods, is_obs=1, dump_at=(), dump_base=0):
        da = np.ascontiguousarray(dump_at, np.int32)
        self._chk(N.lib().qjx_run_periods(self.h, n_periods, is_obs, N.ip(da) if da.size else None, int(da.size),
                                          dump_base), "qjx_run_periods")

    def reset_times(self):
        self._chk(N.lib().qjx_reset_times(self.h), "qjx_reset_times")

    def observe(self, dump, is_start=False):
        self._chk(N.lib().qjx_observe(self.h, dump, int(is_start)), "qjx_observe")

    def observables(self, dump0=0, n_dumps=1, want_adr=False):
        n = self.n
        out = {k: np.zeros((n_dumps, n)) for k in ("norm", "mean", "dispersion", "m2", "energy")}
        robs = np.zeros((n_dumps, n, max(self.nr, 1)), np.complex128)
        adr = None
        if want_adr:
            adr = np.zeros((n_dumps, n, self.d)) if self.keep_adr else np.zeros((n, self.d))
        self._chk(N.lib().qjx_get_observables(self.h, dump0, n_dumps, N.dp(out["norm"]), N.dp(out["mean"]),
                                              N.dp(out["dispersion"]), N.dp(out["m2"]), N.dp(out["energy"]),
                                              N.dp(robs), N.dp(adr)), "qjx_get_observables")
        out["random_obs"] = robs[:, :, : self.nr]
        if want_adr:
            out["adr"] = adr
        return out

    def mean_start(self):
        ms = np.zeros(self.n)
        self._chk(N.lib().qjx_get_mean_start(self.h, N.dp(ms)), "qjx_get_mean_start")
        return ms

    def purity(self, want_rho=False):
        """Ensemble purity Tr(rho^2) of the current states (and rho itself with want_rho)."""
        p = np.zeros(1)
        rho = np.zeros((self.d, self.d), np.complex128) if want_rho else None
        self._chk(N.lib().qjx_purity(self.h, N.dp(p), N.dp(rho)), "qjx_purity")
        return (p[0], rho) if want_rho else p[0]

    def states(self):
        psi = np.zeros((self.n, self.d), np.complex128)
        t = np.zeros(self.n)
        eta = np.zeros(self.n)
        jc = np.zeros(self.n, np.int32)
        self._chk(N.lib().qjx_get_states(self.h, N.dp(psi), N.dp(t), N.dp(eta), N.ip(jc)), "qjx_get_states")
        return psi, t, eta, jc

    def jumps(self, tr):
        k = C.c_int64()
        self._chk(N.lib().qjx_jump_count(self.h, tr, C.byref(k)), "qjx_jump_count")
        k = k.value
        times, norms, etas = np.zeros(k), np.zeros(k), np.zeros(k)
        types = np.zeros(k, np.int32)
        self._chk(N.lib().qjx_get_jumps(self.h, tr, N.dp(times), N.ip(types), N.dp(norms), N.dp(etas)),
                  "qjx_get_jumps")
        return times, types, norms, etas

    def set_active(self, n_active):
        """Later run_periods calls advance trajectories [0, n_active) only."""
        self._chk(N.lib().qjx_set_active(self.h, int(n_active)), "qjx_set_active")

    def set_bases_only(self, on=True):
        """Later run_periods calls advance the Lyapunov bases of every ensemble only."""
        self._chk(N.lib().qjx_set_bases_only(self.h, int(on)), "qjx_set_bases_only")

    # ---------------------------------------------------------- Lyapunov task (task_id 7)
    def lpn_start(self, lpn_type=-1, eps_deep=100, eps_low=-10.0, eps_high=10.0, eps_error=1e-10, delta_s=1e-3,
                  delta_f_high=1e-1, delta_f_low=1e-5, per_period=0, max_energy=1.0, mbl_Nc=0, spec_div=1.0,
                  chars_sys=None):
        """Copy every base [0, n/2) into its variation n/2 + b and perturb it (LpnMult trans_process);
        keyword names follow the reference's lpn_* params.  mbl_Nc > 0 selects the MBL
        characteristics (H in observable slot 0, spec = slot 0 / spec_div, mean = imbalance); chars_sys
        1 the JCS ones (a in slot 0, spec = slot 0 / alpha, mean = <a^+ a> from the energy
        observable), 5 the Integrable ones (the special matrix in slot 0, spec_div 1)."""
        c = N.QjxLpnConfig(lpn_type=lpn_type, eps_deep=eps_deep, per_period=int(per_period), eps_low=eps_low,
                           eps_high=eps_high, eps_error=eps_error, delta_s=delta_s, delta_f_high=delta_f_high,
                           delta_f_low=delta_f_low, max_energy=max_energy, mbl_Nc=mbl_Nc, spec_div=spec_div,
                           chars_sys=(3 if mbl_Nc else 0) if chars_sys is None else chars_sys)
        self._chk(N.lib().qjx_lpn_start(self.h, C.byref(c)), "qjx_lpn_start")

    def lpn_period(self, curr_time, adr_dump=-1):
        """calc_chars_lpn of the bases and lambda_lpn of the variations after one period."""
        self._chk(N.lib().qjx_lpn_period(self.h, float(curr_time), int(adr_dump)), "qjx_lpn_period")

    def lpn_bases(self):
        """calc_chars_lpn of the bases only (LpnMultDeep sub-periods without a Lyapunov step)."""
        self._chk(N.lib().qjx_lpn_bases(self.h), "qjx_lpn_bases")

    def run_sub_periods(self, n_sub, dump_base=0):
        """Deep tasks: continue every trajectory for n_sub sub-periods, observables after each."""
        self._chk(N.lib().qjx_run_sub_periods(self.h, int(n_sub), int(dump_base)), "qjx_run_sub_periods")

    def lpn_values(self):
        n = self.n
        out = {k: np.zeros(n) for k in ("lambda_now", "lambda", "delta_s", "mean_lpn", "energy_lpn")}
        robs = np.zeros((n, max(self.nr, 1)), np.complex128)
        nr = np.zeros(n, np.int32)
        self._chk(N.lib().qjx_lpn_get(self.h, N.dp(out["lambda_now"]), N.dp(out["lambda"]), N.dp(out["delta_s"]),
                                      N.dp(out["mean_lpn"]), N.dp(out["energy_lpn"]), N.dp(robs), N.ip(nr)),
                  "qjx_lpn_get")
        out["robs_lpn"] = robs[:, : self.nr]
        out["num_renorms"] = nr
        return out

    def lpn_last(self):
        n = self.n
        ren, it = np.zeros(n, np.int32), np.zeros(n, np.int32)
        out = {k: np.zeros(n) for k in ("ratio", "delta_s", "delta_f", "eps")}
        self._chk(N.lib().qjx_lpn_get_last(self.h, N.ip(ren), N.dp(out["ratio"]), N.dp(out["delta_s"]),
                                           N.dp(out["delta_f"]), N.ip(it), N.dp(out["eps"])), "qjx_lpn_get_last")
        out["renormed"] = ren
        out["eps_iters"] = it
        return out

    def checkpoint(self, out=None):
        """The engine's complete trajectory state (qjx_checkpoint_save): bytes, or written into the
        caller's uint8 numpy array `out` (e.g. pinned host memory) and returned as its used prefix."""
        size = C.c_size_t()
        self._chk(N.lib().qjx_checkpoint_size(self.h, C.byref(size)), "qjx_checkpoint_size")
        if out is not None:
            if out.dtype != np.uint8 or out.nbytes < size.value or not out.flags["C_CONTIGUOUS"]:
                raise ValueError(f"checkpoint needs a contiguous uint8 buffer of {size.value} bytes")
            self._chk(N.lib().qjx_checkpoint_save(self.h, out.ctypes.data_as(C.c_void_p), size.value),
                      "qjx_checkpoint_save")
            return out[: size.value]
        buf = C.create_string_buffer(size.value)
        self._chk(N.lib().qjx_checkpoint_save(self.h, buf, size.value), "qjx_checkpoint_save")
        return buf.raw

    def checkpoint_size(self):
        size = C.c_size_t()
        self._chk(N.lib().qjx_checkpoint_size(self.h, C.byref(size)), "qjx_checkpoint_size")
        return size.value

    def restore(self, blob):
        """Continue from a checkpoint of an engine with the same configuration (bytes, or a uint8
        numpy array such as a pinned host buffer)."""
        if isinstance(blob, np.ndarray):
            blob = np.ascontiguousarray(blob, np.uint8)
            self._chk(N.lib().qjx_checkpoint_load(self.h, blob.ctypes.data_as(C.c_void_p), blob.nbytes),
                      "qjx_checkpoint_load")
            return
        buf = C.create_string_buffer(blob, len(blob))
        self._chk(N.lib().qjx_checkpoint_load(self.h, buf, len(blob)), "qjx_checkpoint_load")

    def set_trace(self, enable=True):
        self._chk(N.lib().qjx_set_trace(self.h, int(enable)), "qjx_set_trace")

    def trace(self):
        """Per-CTA accumulated trace: columns total, setup, reserved, loop, epilogue cycles,
        sub-tiles, 8-column blocks, columns."""
        nc, nf = C.c_int(), C.c_int()
        self._chk(N.lib().qjx_get_trace(self.h, None, C.byref(nc), C.byref(nf)), "qjx_get_trace")
        out = np.zeros((nc.value, nf.value), np.int64)
        self._chk(N.lib().qjx_get_trace(self.h, out.ctypes.data_as(N.c_i64_p), C.byref(nc), C.byref(nf)),
                  "qjx_get_trace")
        return out

    def device_bytes(self):
        """Device memory this engine holds (qjx_engine_bytes)."""
        b = C.c_size_t()
        self._chk(N.lib().qjx_engine_bytes(self.h, C.byref(b)), "qjx_engine_bytes")
        return b.value

    def stats(self):
        s = N.QjxStats()
        self._chk(N.lib().qjx_get_stats(self.h, C.byref(s)), "qjx_get_stats")
        return {k: getattr(s, k) for k, _ in N.QjxStats._fields_}


def fbasis_pure_state(N, k):
    """f-vector of rho = |k><k| (initRhoODE, source/cpp/CQdiss_os_dimer/CQdiss/calcODE.cpp:120-167):
    only the diagonal generalised Gell-Mann coordinates are nonzero."""
    d = N + 1
    x = np.zeros(d * d - 1)
    base = d * (d - 1)
    for m in range(N):
        w = 1.0 / np.sqrt((m + 1) * (m + 2))
        x[base + m] = w * (1.0 if k <= m else 0.0) - w * (m + 1) * (1.0 if k == m + 1 else 0.0)
    return x


class FBasis:
    """f-basis RK4 of dx/dt = Gs x + E(t) Qs_drv x - Ks on a GPU."""

    def __init__(self, Gs, Qs, Ks, x0, drv_ampl, drv_freq=1.0, drv_phase=0.0, drv_type=0, T=2 * np.pi,
                 num_steps=1000, device=0):
        n = Gs.shape[0]
        self.n = n
        self._keep = []

        def csr(M):
            M = M.tocsr()
            M.sort_indices()
            a = (np.ascontiguousarray(M.indptr, np.int32), np.ascontiguousarray(M.indices, np.int32),
                 np.ascontiguousarray(M.data, np.float64))
            self._keep.append(a)
            return a

        gr, gc, gv = csr(Gs)
        qr, qc, qv = csr(Qs)
        Ks = np.ascontiguousarray(Ks, np.float64)
        x0 = np.ascontiguousarray(x0, np.float64)
        h = C.c_void_p()
        N.check(N.lib().qjx_fb_create(n, N.ip(gr), N.ip(gc), N.dp(gv), N.ip(qr), N.ip(qc), N.dp(qv), N.dp(Ks),
                                      N.dp(x0), drv_ampl, drv_freq, drv_phase, drv_type, T, num_steps, device,
                                      C.byref(h)), what="qjx_fb_create")
        self.h = h

    def run(self, period0, n_periods):
        N.check(N.lib().qjx_fb_run(self.h, period0, n_periods), what="qjx_fb_run")

    def cluster_size(self):
        """CTAs of the cluster-resident RK4 path (0: per-stage kernels)."""
        cs = C.c_int()
        N.check(N.lib().qjx_fb_info(self.h, C.byref(cs)), what="qjx_fb_info")
        return cs.value

    def get(self):
        x = np.zeros(self.n)
        ms = C.c_double()
        N.check(N.lib().qjx_fb_get(self.h, N.dp(x), C.byref(ms)), what="qjx_fb_get")
        return x, ms.value

    def close(self):
        if self.h:
            N.lib().qjx_fb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(U, L, g, HE, T=2 * np.pi, n_traj=2048, precision=0, n_periods=2, seed=0, device=0):
    """Times the candidate tile shapes of one dimension and precision (qjx_autotune) and caches the
    fastest for later engines.  Returns (best, [(tiles, microseconds per trajectory-period)])."""
    U = np.ascontiguousarray(U, np.complex128)
    nb, deep, d, _ = U.shape
    L = np.ascontiguousarray(L, np.complex128).reshape(-1, d, d)
    g = np.ascontiguousarray(np.atleast_1d(g), np.float64)
    HE = np.ascontiguousarray(HE, np.complex128)
    cfg = N.QjxConfig()
    cfg.d, cfg.n_traj, cfg.deep, cfg.num_branches = d, n_traj, deep, nb
    cfg.num_diss, cfg.T, cfg.seed, cfg.device, cfg.precision = L.shape[0], T, seed, device, precision
    cfg.rec_cap, cfg.max_dumps = 16, 1
    best = N.QjxTiles()
    cap = 32
    cand = (N.QjxTiles * cap)()
    us = np.zeros(cap)
    nc = C.c_int(cap)
    N.check(N.lib().qjx_autotune(C.byref(cfg), N.dp(U), N.dp(L), N.dp(g), N.dp(HE), n_periods, C.byref(best), cand,
                                 N.dp(us), C.byref(nc)), what="qjx_autotune")

    def as_dict(t):
        return {k: getattr(t, k) for k, _ in N.QjxTiles._fields_}

    return as_dict(best), [(as_dict(cand[i]), float(us[i])) for i in range(nc.value)]
