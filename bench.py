#!/usr/bin/env python
"""Benchmark of the QJ trajectory engine on one node.

Workload: the driven dissipative Bose dimer at N = 200 (Hilbert dim 201), 10^4 trajectories
per GPU, ex_deep 16, QJ propagator, complex FP64 end to end (the plain drop-in form), Philox
thresholds seed 7, start state |N,0>.  Metric: trajectory-periods per second over all GPUs.

Protocol (the same window in every arm): W untimed warm-up steps of P periods each carry the
ensemble from |N,0> through its transient (periods 1 .. W P); the state at that point is
checkpointed, and each of the K timed steps restores it and runs periods W P + 1 .. W P + P, with
the observables at the end.  `value` is device time of those runs; `e2e` times the same window
through the C ABI from pinned host memory (checkpoint load, run, observables and states read
back); the CPU baseline and the reference arm run the CPU restatement over the same periods on a
sample of the same trajectories (their Philox streams, hence their paths, are the GPU's).

  python bench.py --gpus N --steps K --warmup W            # this engine
  python bench.py --impl reference --steps K --warmup W    # CPU restatement of the reference

Multi-GPU: one process per GPU (torchrun); trajectories are sharded (rank r owns global
trajectories r*n .. r*n+n-1, so the ensemble is the one a single GPU would run), the
ensemble sums of the observables are all-reduced over NCCL once per step.

The same protocol then times the split-precision form (tcgen05 matvecs, FP64 states and norms)
from the same checkpoint; it is reported beside the plain form as "split_form" with its speed-up
and its deviation from the plain form against the horizon.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BOSONS = 200
PRM = dict(J=1.0, U=0.5, E=1.0, A=1.5, g=0.1, omega=1.0)
DEEP = 16
SEED = 7
METRIC = "traj*periods/s"
WORKLOAD = ("dimer N=200 (dim 201), ex_deep 16, QJ propagator, complex FP64 plain form, "
            "10^4 trajectories per GPU x 10 periods per step")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n-traj", type=int, default=10000)
    ap.add_argument("--periods-per-step", type=int, default=10)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-split", action="store_true", help="skip the split-precision form")
    ap.add_argument("--no-fbasis", action="store_true", help="skip the f-basis Lindblad RK4 measurement")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched uneven-ensembles measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop measurement")
    ap.add_argument("--production-sweep", type=int, default=0,
                    help="only time this many points of the N=500 LpnMult production sweep (separate JSON line)")
    ap.add_argument("--serve-window", type=float, default=1.0, help="seconds of Poisson arrivals at 50/s")
    ap.add_argument("--batch-ensembles", type=int, default=32,
                    help="ensembles of the 256-ensemble uneven sweep in the batched measurement")
    ap.add_argument("--profile", action="store_true", help="short run for ncu captures (no JSON line)")
    ap.add_argument("--profile-target", default="plain",
                    choices=["plain", "split", "fbasis", "fbstages", "lpn", "purity", "rk", "batched"],
                    help="what --profile runs: one period of the plain or split form, one f-basis period "
                         "(cluster kernel, or the per-stage kernels), the Lyapunov pair case, ensemble purity, "
                         "the RK propagator or the batched engine")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def model(impl="ours"):
    """Operators of the workload: the library's builder, or for the reference arm the CPU
    restatement's (bit-identical to each other; the reference arm loads no library of ours)."""
    T = 2.0 * 3.1415926535897932384626433832795 / PRM["omega"]
    if impl == "reference":
        from oracle import oracle_py as O

        H, Hd, L, K0, K1 = O.dimer_operators(N_BOSONS, PRM["J"], PRM["U"], PRM["E"], PRM["A"], PRM["g"])
        Ut = np.stack([O.split_tree(K0, T, DEEP), O.split_tree(K1, T, DEEP)])
    else:
        import os_d_b200 as q

        H, Hd, L, Ut = q.build_dimer(N_BOSONS, PRM["J"], PRM["U"], PRM["E"], PRM["A"], PRM["g"], PRM["omega"], DEEP)
    d = N_BOSONS + 1
    HE = H + PRM["E"] * Hd
    rng = np.random.default_rng(1)  # one random observable X X^H / (tr/d)
    X = 0.5 * (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d)))
    R = X @ X.conj().T
    R = (R / (np.trace(R).real / d))[None]
    return dict(H=H, Hd=Hd, L=L, U=Ut, HE=HE, R=R, T=T, d=d)


def bench_config(world, n, d, P, W):
    return {"workload": WORKLOAD, "n_traj_per_gpu": n, "dim": d, "ex_deep": DEEP, "periods_per_step": P,
            "window": f"periods {W * P + 1}..{W * P + P} (after a {W * P}-period transient from |N,0>)",
            "seed": SEED, "start": "|N,0>", "parallelism": f"dp{world} (trajectories)",
            "l2": "flushed between timed steps (256 MB write)"}


def kernel_name(d):
    """Instantiation qjx::step_kernel<NRB, CBMAX> the library picks for dimension d <= 208
    (32-column sub-tiles: CBMAX 4, NRB row blocks per warp at 4 warps per column block)."""
    rb = (d + 7) // 8
    return f"qjx::step_kernel<{(rb + 3) // 4}, 4>"


def start_states(n, d):
    psi = np.zeros((n, d), np.complex128)
    psi[:, 0] = 1.0
    return psi


# ---------------------------------------------------------------- CPU restatement (baseline)
CPU_STATE = ("phi", "eta", "t", "rng_pos", "jumps_counts", "n_rec", "error")


def cpu_windows(M, n_traj, threads, warm_periods, P, windows):
    """The CPU restatement (oracle/qjx_oracle.c, OpenMP over trajectories like the reference,
    QJX/experiment.cpp:484) on trajectories 0 .. n_traj - 1 of the benchmark ensemble: an untimed
    transient of warm_periods periods, then `windows` timed runs of the next P periods, each from
    the state the transient left.  Returns [(traj*periods/s, seconds, matvecs per traj*period)]."""
    from oracle import oracle_py as O

    ens = O.Ensemble(M["U"], M["L"], [1.0], M["HE"], M["R"], M["T"], n_traj, seed=SEED, record=0)
    ens.init(0, 0)
    if warm_periods and ens.run_periods(warm_periods, is_obs=1, n_threads=threads):
        raise RuntimeError("oracle reported trajectory errors")
    snap = {k: getattr(ens, k).copy() for k in CPU_STATE}
    out = []
    for _ in range(windows):
        for k, v in snap.items():
            getattr(ens, k)[...] = v
        mv0 = int(ens.matvecs.sum())
        t0 = time.perf_counter()
        bad = ens.run_periods(P, is_obs=1, n_threads=threads)
        dt = time.perf_counter() - t0
        if bad:
            raise RuntimeError("oracle reported trajectory errors")
        out.append((n_traj * P / dt, dt, (int(ens.matvecs.sum()) - mv0) / (n_traj * P)))
    return out


CPU_TRAJ_PER_THREAD = 3


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    M = model("reference")
    threads = os.cpu_count() or 1
    sample = CPU_TRAJ_PER_THREAD * threads
    P = args.periods_per_step
    res = cpu_windows(M, sample, threads, args.warmup * P, P, args.steps)
    value = float(np.mean([r[0] for r in res]))
    tot = sum(r[1] for r in res)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(args.gpus, args.n_traj, M["d"], P, args.warmup),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": (f"trajectories 0..{sample - 1} of the ensemble (their paths are the GPU's), "
                                    f"the same {P}-period window after the same {args.warmup * P}-period transient, "
                                    f"OpenMP over trajectories on {threads} host threads")},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("the reference (source/cpp/QJX) needs Intel MKL and Eigen, absent here; this arm times the "
                 "C restatement of its algorithm (oracle/qjx_oracle.c) on the host cores, with operators from "
                 "oracle/oracle_py.py (no library of this repository is loaded)"),
        "matvecs_per_traj_period": float(np.mean([r[2] for r in res])),
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- f-basis Lindblad RK4 (dimer N = 50, dt = 1e-3)
FB_N, FB_DT, FB_A = 50, 1e-3, 1.5


def fbasis_bench(args, local):
    """The density-matrix oracle path: dimer N = 50 (f-vector of 2600), RK4 with dt = 1e-3
    (6284 steps per period), one period per step; device time of qjx_fb_run."""
    import math

    import scipy.sparse as sp

    import os_d_b200 as q
    from os_d_b200 import _native as Nt

    (gr, gc, gv), (qr, qc, qv), ks = Nt.fb_build_dimer(FB_N, PRM["J"], PRM["U"], PRM["E"], PRM["g"])
    n = ks.size
    Gs = sp.csr_matrix((gv, gc, gr), shape=(n, n))
    Qs = sp.csr_matrix((qv, qc, qr), shape=(n, n))
    T = 2.0 * math.pi
    steps = math.ceil(T / FB_DT)
    fb = q.FBasis(Gs, Qs, ks, q.fbasis_pure_state(FB_N, 0), FB_A, T=T, num_steps=steps, device=local)
    for w in range(args.warmup):
        fb.run(w, 1)
    ms = []
    for k in range(args.steps):
        fb.run(args.warmup + k, 1)
        ms.append(fb.get()[1])
    x = fb.get()[0]
    cs = fb.cluster_size()
    fb.close()
    per = float(np.mean(ms))
    nnz = Gs.nnz + Qs.nnz
    step_bytes = 4 * (12.0 * nnz + 24.0 * n)  # CSR operands + stage vectors, 4 stages
    achieved = step_bytes * steps / (per * 1e-3) / 1e9
    smem_peak = (cs if cs else 1) * 128 * 1.965e9 / 1e9
    out = {"workload": f"f-basis Lindblad RK4, dimer N={FB_N} (f-vector {n}), dt={FB_DT} ({steps} steps/period), "
                       f"Gs nnz {Gs.nnz}, Qs nnz {Qs.nnz}",
           "metric": "periods/s", "value": 1e3 / per, "ms_per_period": per, "us_per_rk4_step": 1e3 * per / steps,
           "kernel": "fb::rk4_cluster" if cs else "fb::rk_stage + fb::rk_update", "cluster_size": cs,
           "roofline": {"bound": "shared memory / cluster barrier latency (operands resident in the cluster's shared "
                                 "memory, no HBM traffic after the first load)",
                        "achieved": achieved, "unit": "GB/s", "peak": smem_peak,
                        "peak_source": "shared-memory bandwidth of the cluster's SMs, 128 B/clk at 1965 MHz",
                        "frac": achieved / smem_peak, "algorithmic_bytes_per_rk4_step": step_bytes},
           "purity": float(1.0 / (FB_N + 1) + x @ x)}
    if not args.no_cpu_baseline:
        from oracle import oracle_py as O

        csteps = 200
        t0 = time.perf_counter()
        O.fb_rk4(Gs, Qs, ks, q.fbasis_pure_state(FB_N, 0), FB_A, T=T, num_steps=csteps, n_periods=1)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 1.0 / (dt * steps / csteps), "unit": "periods/s", "cores": 1, "kind": "port",
                               "sample": f"{csteps} RK4 steps of the same system ({dt:.2f} s), "
                                         f"oracle/fbasis_oracle.c, scaled to {steps} steps per period"}
    return out


# ---------------------------------------------------------------- batched uneven ensembles (256 dimers, N ~ U[50, 400])
BATCH_SEED, BATCH_TRAJ = 11, 1000


def batch_draw(count):
    """The uneven sweep's ensembles: N ~ U[50, 400], E0 ~ U[0, 2], g log-uniform in [0.01, 1], seed 11
    (the first `count` of the 256 draws)."""
    rng = np.random.default_rng(BATCH_SEED)
    Ns = rng.integers(50, 401, size=256)
    E0 = rng.uniform(0.0, 2.0, size=256)
    g = 10.0 ** rng.uniform(-2.0, 0.0, size=256)
    return [(int(Ns[i]), float(E0[i]), float(g[i])) for i in range(count)]


def batched_bench(args, local):
    """Chosen form 2: ensembles of uneven dimension advanced together by one engine (one set of
    persistent micro-step launches, CUDA graphs of 6 micro-steps), one period per step, against
    the same ensembles solved one after another by single-ensemble engines (serial plain FP64)."""
    import torch

    import os_d_b200 as q

    ens = []
    t_build = time.perf_counter()
    for i, (N, E0, g) in enumerate(batch_draw(args.batch_ensembles)):
        H, Hd, L, Ut = q.build_dimer(N, PRM["J"], PRM["U"], E0, PRM["A"], g, PRM["omega"], DEEP)
        ens.append(dict(U=Ut, L=L, g=[1.0], HE=H + E0 * Hd, n_traj=BATCH_TRAJ, T=2.0 * np.pi / PRM["omega"],
                        seed=BATCH_SEED, tr_base=i * BATCH_TRAJ))
    t_build = time.perf_counter() - t_build
    dims = [x["U"].shape[-1] for x in ens]
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def prepare(eng, n, rows):
        psi = np.zeros((n, rows), np.complex128)
        psi[:, 0] = 1.0
        eng.set_states(psi)
        eng.init_thresholds()
        eng.reset_times()
        return eng

    B = prepare(q.Engine.batch(ens, deep=DEEP, device=local), BATCH_TRAJ * len(ens), max(dims))
    for _ in range(args.warmup):
        B.run_periods(1, is_obs=1)
    ms, m0 = 0.0, B.stats()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        B.run_periods(1, is_obs=1)
        ms += B.stats()["last_call_ms"]
    m1 = B.stats()
    B.close()
    # serial: each ensemble alone for the same periods; its matvecs give the algorithmic flops
    ms_serial, flops = 0.0, 0.0
    for x in ens:
        d = x["U"].shape[-1]
        A = prepare(q.Engine(x["U"], x["L"], x["g"], x["HE"], None, x["T"], BATCH_TRAJ, seed=x["seed"],
                             tr_base=x["tr_base"], device=local), BATCH_TRAJ, d)
        for _ in range(args.warmup):
            A.run_periods(1, is_obs=1)
        a0 = A.stats()
        for _ in range(args.steps):
            A.run_periods(1, is_obs=1)
            ms_serial += A.stats()["last_call_ms"]
        flops += 8.0 * d * d * (A.stats()["matvecs"] - a0["matvecs"])
        A.close()
    n_tot = BATCH_TRAJ * len(ens)
    kern_s = (m1["step_kernel_ms"] - m0["step_kernel_ms"]) * 1e-3
    peak_ffma, peak_dmma = q.measure_fp64_peak(local)
    peak = max(peak_ffma, peak_dmma)
    # the split form batched: the ensembles of d <= 256 (the tcgen05 N limit), both precisions
    small = [x for x in ens if x["U"].shape[-1] <= 256]
    sub = {}
    for prec in (0, 1):
        E = prepare(q.Engine.batch(small, deep=DEEP, device=local, precision=prec), BATCH_TRAJ * len(small),
                    max(x["U"].shape[-1] for x in small))
        for _ in range(args.warmup):
            E.run_periods(1, is_obs=1)
        ms_p = 0.0
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            E.run_periods(1, is_obs=1)
            ms_p += E.stats()["last_call_ms"]
        sub[prec] = (BATCH_TRAJ * len(small) * args.steps / (ms_p * 1e-3), E.stats().get("rechecks", 0))
        E.close()
    split_batch = {"ensembles": len(small), "dims": [min(x["U"].shape[-1] for x in small),
                                                      max(x["U"].shape[-1] for x in small)],
                   "plain_value": sub[0][0], "split_value": sub[1][0], "split_speedup": sub[1][0] / sub[0][0],
                   "split_rechecks": sub[1][1]}
    return {
        "workload": (f"{len(ens)} of the 256 uneven dimer ensembles (N ~ U[50,400], E0 ~ U[0,2], g log-uniform "
                     f"[0.01,1], seed {BATCH_SEED}; dims {min(dims)}-{max(dims)}), {BATCH_TRAJ} trajectories each, "
                     f"ex_deep {DEEP}, complex FP64, one period per step"),
        "metric": METRIC, "value": n_tot * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps,
        "serial_single_ensemble_engines": {"value": n_tot * args.steps / (ms_serial * 1e-3),
                                           "ms_per_step": ms_serial / args.steps},
        "speedup_vs_serial": ms_serial / ms,
        "roofline": {"bound": "tensor", "kernel": "qjx::step_kernel (per-(ensemble, matrix) buckets)",
                     "achieved": flops / kern_s / 1e12, "peak": peak, "unit": "TFLOP/s",
                     "frac": flops / kern_s / 1e12 / peak,
                     "flops": "8 d_e^2 per executed matvec, summed over the ensembles (matvecs counted by the "
                              "same ensembles run alone, whose trajectories are bit-identical)"},
        "gpu_launches": int(m1["launches"] - m0["launches"]),
        "host_build_s": t_build,
        "split_precision_batch": split_batch,
    }


# ---------------------------------------------------------------- Lyapunov pair kernel (profiling case)
def lpn_profile_case(local):
    """LpnMult on the headline dimer (dim 201): 2000 trajectories (1000 base/variation pairs), the
    bases' transient period, the start (copy + perturbation bisection) and two observation periods
    with lambda_lpn (random-observable distance, renormalisation thresholds of the production sweep
    but delta_f_high = 5e-3 so that pairs renormalise)."""
    import os_d_b200 as q

    M = model()
    n, d = 2000, M["d"]
    eng = q.Engine(M["U"], M["L"], [1.0], M["HE"], M["R"], M["T"], n, seed=SEED, max_dumps=1, device=local)
    eng.set_states(start_states(n, d))
    eng.init_thresholds()
    eng.set_active(n // 2)
    eng.run_periods(1, is_obs=0)
    eng.set_active(n)
    eng.lpn_start(lpn_type=0, eps_deep=100, eps_low=-10.0, eps_high=10.0, eps_error=1e-10, delta_s=1e-3,
                  delta_f_high=5e-3, delta_f_low=1e-5)
    eng.reset_times()
    for p in range(2):
        eng.run_periods(1, is_obs=1)
        eng.lpn_period((p + 1) * M["T"])
    v = eng.lpn_values()
    print(json.dumps({"pairs": n // 2, "renormalisations": int(v["num_renorms"].sum()),
                      "bisection_steps_last": int(eng.lpn_last()["eps_iters"][n // 2:].sum())}), flush=True)
    eng.close()


def profile_case(target, local):
    """Short runs of the kernels outside the headline step, for ncu captures:
    purity  -- dimer dim 201, 10^4 trajectories after one period: normalize, rho and purity kernels
               (three ensemble-purity evaluations with the density matrix);
    rk      -- the RK propagator (prop_id 1) on dim 101 (N = 100, g = 0.4, where 2000 RK4 steps per
               period are stable), 2000 trajectories, one period;
    batched -- the first 8 of the 256 uneven ensembles (1000 trajectories each) in one batched
               engine, one period."""
    import os_d_b200 as q

    if target == "purity":
        M = model()
        n, d = 10000, M["d"]
        eng = q.Engine(M["U"], M["L"], [1.0], M["HE"], M["R"], M["T"], n, seed=SEED, max_dumps=1, device=local)
        eng.set_states(start_states(n, d))
        eng.init_thresholds()
        eng.run_periods(1, is_obs=0)
        for _ in range(3):
            p, _ = eng.purity(want_rho=True)
        print(json.dumps({"purity": p}), flush=True)
        eng.close()
    elif target == "rk":
        N_ = 100
        H, Hd, L, _ = q.build_dimer(N_, PRM["J"], PRM["U"], PRM["E"], PRM["A"], 0.4, PRM["omega"], 1)
        n, d = 2000, N_ + 1
        Lm = np.asarray(L).reshape(d, d)
        Heff = H - 0.5j * (0.4 / N_) * (Lm.conj().T @ Lm)  # the dimer's rate g / N on L^+ L
        eng = q.Engine.rk(Heff, Hd, L, [1.0], H + PRM["E"] * Hd, None, 2.0 * np.pi / PRM["omega"], n, E0=PRM["E"],
                          A=PRM["A"], rk_ns=2000, seed=SEED, max_dumps=1, device=local)
        eng.set_states(start_states(n, d))
        eng.init_thresholds()
        eng.run_periods(1, is_obs=1)
        print(json.dumps({"rk_micro_steps": eng.stats()["micro_steps"]}), flush=True)
        eng.close()
    elif target == "batched":
        ens = []
        for i, (N_, E0, g) in enumerate(batch_draw(8)):
            H, Hd, L, Ut = q.build_dimer(N_, PRM["J"], PRM["U"], E0, PRM["A"], g, PRM["omega"], DEEP)
            ens.append(dict(U=Ut, L=L, g=[1.0], HE=H + E0 * Hd, n_traj=BATCH_TRAJ, T=2.0 * np.pi / PRM["omega"],
                            seed=BATCH_SEED, tr_base=i * BATCH_TRAJ))
        rows = max(x["U"].shape[-1] for x in ens)
        B = q.Engine.batch(ens, deep=DEEP, device=local)
        psi = np.zeros((BATCH_TRAJ * len(ens), rows), np.complex128)
        psi[:, 0] = 1.0
        B.set_states(psi)
        B.init_thresholds()
        B.run_periods(1, is_obs=1)
        print(json.dumps({"batched_micro_steps": B.stats()["micro_steps"]}), flush=True)
        B.close()


# ---------------------------------------------------------------- production Lyapunov sweep (sampled)
def production_sweep(args, local):
    """The reference's production dimer workload (submit/qjx/submit_dimer.py): LpnMult (task_id 7) at
    N = 500 (dim 501), 20 trajectories (10 base/variation pairs) per parameter point, U = 0.01,
    0.02, ..., A = 1.5, E = 1, J = 1, g = 0.1, one random observable (lpn_type 0), ex_deep 16.  The
    first `count` U values run as one batched engine, one observation period (with the Lyapunov
    update) per step, against the same points solved one after another by single-ensemble engines,
    and against the CPU restatement on the host cores."""
    import os_d_b200 as q

    count, n, N = args.production_sweep, 20, 500
    d = N + 1
    R = q.random_observables(d, 1, 100, 1000000, 2)
    cfg = dict(lpn_type=0, eps_deep=100, eps_low=-10.0, eps_high=10.0, eps_error=1e-10, delta_s=1e-3,
               delta_f_high=1e-1, delta_f_low=1e-5)
    t_build = time.perf_counter()
    ens = []
    for i in range(count):
        U = 0.01 * (i + 1)
        H, Hd, L, Ut = q.build_dimer(N, 1.0, U, 1.0, 1.5, 0.1, 1.0, DEEP)
        ens.append(dict(U=Ut, L=L, g=[1.0], HE=H + Hd, R=R, n_traj=n, T=2.0 * np.pi, seed=0, tr_base=0))
    t_build = time.perf_counter() - t_build

    def flow(eng, rows, steps):
        psi = np.zeros((eng.n, rows), np.complex128)
        psi[:, 0] = 1.0
        eng.set_states(psi)
        eng.init_thresholds()
        eng.set_bases_only(True)
        eng.run_periods(1, is_obs=0)  # (a sample of) the bases' transient
        eng.set_bases_only(False)
        eng.lpn_start(**cfg)
        eng.reset_times()
        ms = 0.0
        for p in range(steps):
            eng.run_periods(1, is_obs=1)
            eng.lpn_period((p + 1) * 2.0 * np.pi)
            ms += eng.stats()["last_call_ms"]
        return ms, eng.stats()

    B = q.Engine.batch(ens, deep=DEEP, max_dumps=1, device=local)
    ms_b, st_b = flow(B, d, args.steps)
    v = B.lpn_values()
    B.close()
    ms_s = 0.0
    for x in ens:
        A = q.Engine(x["U"], x["L"], x["g"], x["HE"], x["R"], x["T"], n, seed=0, max_dumps=1, device=local)
        m, _ = flow(A, d, args.steps)
        ms_s += m
        A.close()
    out = {"workload": (f"LpnMult (task_id 7) production sweep sample: {count} parameter points U = 0.01..{0.01 * count:.2f} "
                        f"of submit_dimer.py, dimer N={N} (dim {d}), {n} trajectories each, ex_deep {DEEP}, "
                        f"lpn_type 0, one observation period + Lyapunov update per step"),
           "metric": METRIC, "value": count * n * args.steps / (ms_b * 1e-3), "ms_per_step": ms_b / args.steps,
           "serial_single_ensemble_engines": {"value": count * n * args.steps / (ms_s * 1e-3),
                                              "ms_per_step": ms_s / args.steps},
           "speedup_vs_serial": ms_s / ms_b, "renormalisations": int(v["num_renorms"].sum()),
           "matvecs_per_traj_period": (st_b["matvecs"]) / (count * n * (args.steps + 1)),
           "host_build_s": t_build}
    if not args.no_cpu_baseline:
        from oracle import oracle_py as O

        threads = os.cpu_count() or 1
        x = ens[0]
        o = O.Ensemble(x["U"], x["L"], x["g"], x["HE"], x["R"], x["T"], threads, seed=0, record=0)
        o.init(0, 0)
        t0 = time.perf_counter()
        assert o.run_periods(1, is_obs=1, n_threads=threads) == 0
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": threads / dt, "unit": METRIC, "cores": threads, "kind": "port",
                               "sample": f"{threads} trajectories x 1 period at dim {d} ({dt:.1f} s), oracle/qjx_oracle.c"}
    return out


# ---------------------------------------------------------------- serving loop (requests up to N = 1023, sampled)
def serving_bench(args, local):
    """Continuous batching (os_d_b200.serve): Poisson arrivals at 50/s over a short window with
    the serving workload's size range (N log-uniform in [31, 1023]; E0 ~ U[0, 2], g log-uniform in
    [0.01, 1], seed 23) but trajectories U[10, 1000] and 1-3 periods (its full sizes, up to 10^4
    trajectories x 500 periods at d = 1024, are hours of device time per request); size-class pools
    admitted against the device's free memory, operators built on the GPU; latency from arrival to
    result on the wall clock; the same requests then solved one after another by single-ensemble
    engines (serial plain FP64)."""
    import os_d_b200 as q
    from os_d_b200.serve import Server, dimer_ensemble

    rng = np.random.default_rng(23)
    arrivals, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / 50.0)
        if t > args.serve_window:
            break
        N = int(round(10 ** rng.uniform(np.log10(31), np.log10(1023))))
        arrivals.append((t, dict(N=N, n_traj=int(rng.integers(10, 1001)), periods=int(rng.integers(1, 4)),
                                 E0=float(rng.uniform(0, 2)), g=float(10 ** rng.uniform(-2, 0)), seed=23,
                                 tr_base=1000 * len(arrivals))))
    srv = Server(deep=DEEP, device=local)
    t0 = time.perf_counter()
    res = srv.run(arrivals)
    wall = time.perf_counter() - t0
    dev_ms, pools, peak = srv.device_ms, srv.pools_created, srv.peak_bytes
    srv.close()
    lat = np.array([r["t_done"] - r["t_submit"] for r in res])
    work = float(sum(r["n_traj"] * r["periods"] for r in res))
    # serial plain FP64 solves of the same requests (device time of each alone)
    ser_ms = 0.0
    per_req = []  # (d, n_traj * periods, device ms) of each request alone
    for _, r in arrivals:
        e = dimer_ensemble(r, DEEP, local)
        d, n = e["U"].shape[-1], e["n_traj"]
        A = q.Engine(e["U"], e["L"], e["g"], e["HE"], None, e["T"], n, seed=e["seed"], tr_base=e["tr_base"],
                     max_dumps=1, device=local)
        psi = np.zeros((n, d), np.complex128)
        psi[:, 0] = 1.0
        A.set_states(psi)
        A.init_thresholds()
        A.run_periods(int(r["periods"]), is_obs=1, dump_at=[int(r["periods"])], dump_base=0)
        ser_ms += A.stats()["kernel_ms"]
        per_req.append((d, n * int(r["periods"]), A.stats()["kernel_ms"]))
        A.close()
    # what one GPU sustains at the serving workload's full request sizes: the device time per
    # trajectory-period of a request alone, fitted as a + b d^2 over the sample, averaged over
    # the full request distribution (N log-uniform [31, 1023], trajectories U[100, 10^4], periods
    # U[50, 500]), and divided by the serving loop's measured gain over serial solves
    dd = np.array([x[0] for x in per_req], float)
    tp = np.array([x[1] for x in per_req], float)
    ms = np.array([x[2] for x in per_req], float)
    A_ = np.stack([tp, tp * dd * dd], axis=1)
    coef = np.linalg.lstsq(A_, ms, rcond=None)[0]
    rng5 = np.random.default_rng(5)
    N5 = np.round(10 ** rng5.uniform(np.log10(31), np.log10(1023), 100000))
    d5 = N5 + 1
    req_ms = (rng5.uniform(100, 1e4, 100000) * rng5.uniform(50, 500, 100000)) * (coef[0] + coef[1] * d5 * d5)
    gain = max(ser_ms / dev_ms, 1e-9)
    sustain = 1e3 * gain / float(req_ms.mean())
    return {
        "workload": (f"{len(arrivals)} requests, Poisson 50/s over {args.serve_window:g} s; dimer N log-uniform "
                     f"[31,1023] (d up to 1024), trajectories U[10,1000], periods U[1,3], E0 ~ U[0,2], g log-uniform "
                     f"[0.01,1], seed 23; size-class pools of 8 slots admitted against free device memory"),
        "metric": METRIC, "value": work / wall, "device_value": work / (dev_ms * 1e-3),
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "max": float(lat.max())},
        "serial_single_ensemble_engines": {"value": work / (ser_ms * 1e-3), "device_s": ser_ms * 1e-3},
        "speedup_vs_serial_device": ser_ms / dev_ms, "pools_created": pools, "peak_pool_bytes": peak,
        "wall_s": wall, "max_d": int(max(r["N"] for _, r in arrivals)) + 1,
        "full_size_sustained": {
            "requests_per_s": sustain, "mean_request_device_s": float(req_ms.mean()) * 1e-3 / gain,
            "model": "device ms of a request alone = trajectory-periods x (a + b d^2), fitted over this sample "
                     f"(a = {coef[0]:.3g}, b = {coef[1]:.3g}); averaged over the full request sizes (N log-uniform "
                     "[31,1023], trajectories U[100,10^4], periods U[50,500]) and divided by the serving loop's "
                     "measured gain over serial solves; an arrival rate of 50 requests/s exceeds it by the ratio"},
    }


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.gpu = gpu_index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-i", str(self.gpu), "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for row in self.f.read().strip().splitlines():
            c = [x.strip() for x in row.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                smax.append(float(c[2]))
            except ValueError:
                continue
            for nm, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- split-precision form
def split_form(args, q, new_engine, timed_windows, snap, value, ens_plain, x_plain, eng_plain, n, d, P, W, world):
    """The split-precision form (precision 1) from the same checkpoint over the same windows, its
    speed-up over the plain form, and its deviation from the plain form against the horizon: one
    more window of both forms with the observables after every period."""
    eng_s = new_engine(1)
    ms_s, _, _, s0, s1, ens_split, x_split = timed_windows(eng_s, snap)
    v_s = world * n * P * args.steps / (ms_s * 1e-3)
    tiles = s1["mma_tiles"] - s0["mma_tiles"]
    mds, ks = 16 * ((d + 15) // 16), (d + 15) // 16
    exec_flops = tiles * ks * 12 * 2.0 * 128 * mds * 16
    kern_s = (s1["step_kernel_ms"] - s0["step_kernel_ms"]) * 1e-3
    peaks = {}
    pk_file = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_file):
        with open(pk_file) as f:
            peaks = json.load(f)
    bf16_peak = peaks.get("bf16_tflops", 1590.0)
    # horizon: observables after each of the P periods of one more window, both forms
    base = W + args.steps + 1
    per_period = {}
    for name, e in (("plain", eng_plain), ("split", eng_s)):
        e.restore(snap)
        e.run_periods(P, is_obs=1, dump_at=list(range(1, P + 1)), dump_base=base)
        ob = e.observables(base, P)
        per_period[name] = (N_BOSONS - 2.0 * ob["mean"], ob["energy"])
        per_period[name + "_jumps"] = e.states()[3]
    hor = []
    for h in range(P):
        xp, xs = per_period["plain"][0][h], per_period["split"][0][h]
        ep, es = per_period["plain"][1][h], per_period["split"][1][h]
        same = np.abs(xs - xp) < 1e-3  # an identical jump path leaves only the matvec rounding
        hor.append({"periods": h + 1,
                    "n1_minus_n2_abs_diff": float(abs(xs.mean() - xp.mean())),
                    "n1_minus_n2_stderr": float(xp.std() / np.sqrt(xp.size)),
                    "energy_abs_diff": float(abs(es.mean() - ep.mean())),
                    "same_path_fraction": float(same.mean()),
                    "max_abs_diff_on_same_paths": float(np.abs(xs - xp)[same].max()) if same.any() else None})
    eng_s.close()
    # speed against accuracy: the recheck band is the knob (off, the default 1e-5, wider; a band
    # of 1 rechecks every norm test, which makes the split form bit-identical to the plain one)
    HC = 2
    eng_plain.restore(snap)
    eng_plain.run_periods(HC, is_obs=1, dump_at=list(range(1, HC + 1)), dump_base=base)
    ms_plain_hc = eng_plain.stats()["last_call_ms"]
    xp_hc = N_BOSONS - 2.0 * eng_plain.observables(base, HC)["mean"]
    curve = []
    for band in (-1.0, 1e-5, 1e-4, 1e-3, 1e-2, 1.0):
        e = new_engine(1, split_recheck=band)
        e.restore(snap)
        r0 = e.stats()["rechecks"]
        e.run_periods(HC, is_obs=1, dump_at=list(range(1, HC + 1)), dump_base=base)
        ms_b = e.stats()["last_call_ms"]
        xs_hc = N_BOSONS - 2.0 * e.observables(base, HC)["mean"]
        curve.append({"split_recheck": band if band > 0 else "off",
                      "speedup_vs_plain": ms_plain_hc / ms_b,
                      "rechecks_per_traj_period": (e.stats()["rechecks"] - r0) / (n * HC),
                      "same_path_fraction": [float(np.mean(np.abs(xs_hc[h] - xp_hc[h]) < 1e-3)) for h in range(HC)],
                      "n1_minus_n2_abs_diff": [float(abs(xs_hc[h].mean() - xp_hc[h].mean())) for h in range(HC)]})
        e.close()
    return {
        "metric": METRIC, "value": v_s, "unit": METRIC, "ms_per_step": ms_s / args.steps,
        "speedup_vs_plain": v_s / value,
        "dtype": "bf16x3 matvec on tcgen05 (FP32 accumulate), FP64 states, norms, decisions and observables",
        "n1_minus_n2_abs_diff_vs_plain_per_step": [abs(a[0] - b[0]) for a, b in zip(ens_split, ens_plain)],
        "n1_minus_n2_stderr_per_step": [b[1] for b in ens_plain],
        "same_jump_count_fraction_after_window": float(np.mean(per_period["split_jumps"] == per_period["plain_jumps"])),
        "horizon": hor,
        "recheck_curve": {"periods": HC, "window_start": "the timed window's checkpoint", "points": curve},
        "roofline": {"bound": "tensor", "kernel": "qjx::split_step_kernel",
                     "achieved": exec_flops / kern_s / 1e12, "peak": bf16_peak, "unit": "TFLOP/s",
                     "frac": exec_flops / kern_s / 1e12 / bf16_peak,
                     "peak_source": "MEASURED_PEAKS.json bf16_tflops (cuBLAS bf16 burst)" if peaks else "fallback 1590",
                     "flops": "executed tcgen05 bf16 flops: 12 MMAs of 128 x MDs x 16 per k-step and tile",
                     "algorithmic_tflops": 8.0 * d * d * (s1["matvecs"] - s0["matvecs"]) / kern_s / 1e12},
        "matvecs_per_traj_period": (s1["matvecs"] - s0["matvecs"]) / (n * P * args.steps),
        "gpu_launches": int(s1["launches"] - s0["launches"]),
    }


# ---------------------------------------------------------------- this engine
def run_ours(args):
    import torch

    import os_d_b200 as q

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        pg = dist

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    def allreduce(x, op="sum"):
        t = torch.tensor(x, dtype=torch.float64, device="cuda")
        if pg:
            pg.all_reduce(t, op=pg.ReduceOp.MAX if op == "max" else pg.ReduceOp.SUM)
        return t.cpu().numpy()

    M = model()
    n, d, P, W = args.n_traj, M["d"], args.periods_per_step, args.warmup
    tuned = None
    if not args.profile and args.production_sweep == 0:
        # the project's autotuner picks the tile shapes of this dimension in both precisions (cached
        # for the engines below in a file of this run)
        os.environ.setdefault("QJX_TILE_CACHE", os.path.join(tempfile.mkdtemp(), "tiles.txt"))
        tuned = {}
        for prec in (0, 1):
            best, table = q.autotune(M["U"], M["L"], [1.0], M["HE"], T=M["T"], n_traj=2048, precision=prec,
                                     n_periods=1, device=local)
            tuned["split" if prec else "plain"] = {"best": best, "candidates_us_per_traj_period":
                                                   [[t, round(us, 4)] for t, us in table]}
    steps_total = W + args.steps
    psi0 = start_states(n, d)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def new_engine(precision, split_recheck=0.0):
        e = q.Engine(M["U"], M["L"], [1.0], M["HE"], M["R"], M["T"], n, seed=SEED, record=0, rec_cap=16,
                     keep_adr=0, max_dumps=steps_total + P + 2, device=local, tr_base=rank * n, precision=precision,
                     split_recheck=split_recheck)
        e.set_states(psi0)
        e.init_thresholds()
        e.reset_times()
        e.observe(0, is_start=True)
        return e

    def n1n2(eng, slot):
        return N_BOSONS - 2.0 * eng.observables(slot, 1)["mean"][0]

    def ensemble(x):
        """ensemble mean of <n1 - n2> and its standard error; the sums are reduced over ranks
        (the one exchange of the path)"""
        s = allreduce([float(np.sum(x)), float(np.sum(x * x)), float(x.size)])
        m = s[0] / s[2]
        return m, float(np.sqrt(max(s[1] / s[2] - m * m, 0.0) / s[2]))

    def timed_windows(eng, snap, clocks=None):
        """K timed runs of the window, each from the checkpoint `snap`; device time of each run
        (CUDA events around the micro-step launches), max over ranks."""
        st0 = eng.stats()
        barrier()
        if clocks:
            clocks.start()
        t0 = time.perf_counter()
        dev_ms, ens, x_last = 0.0, [], None
        for k in range(args.steps):
            eng.restore(snap)
            flush.zero_()  # L2 flush between timed steps
            torch.cuda.synchronize()
            slot = 1 + W + k
            eng.run_periods(P, is_obs=1, dump_at=[P], dump_base=slot)
            dev_ms += eng.stats()["last_call_ms"]
            x_last = n1n2(eng, slot)
            ens.append(ensemble(x_last))
        barrier()
        wall = time.perf_counter() - t0
        clk = clocks.stop() if clocks else None
        return float(allreduce([dev_ms], "max")[0]), wall, clk, st0, eng.stats(), ens, x_last

    if args.production_sweep > 0:
        if rank == 0:
            print(json.dumps({"production_sweep": production_sweep(args, local)}), flush=True)
        return
    if args.profile and args.profile_target == "lpn":
        lpn_profile_case(local)
        return
    if args.profile and args.profile_target in ("fbasis", "fbstages"):
        if args.profile_target == "fbstages":
            os.environ["QJX_FB_PATH"] = "stages"
        args.warmup, args.steps, args.no_cpu_baseline = 0, 1, True
        print(json.dumps({"fbasis": fbasis_bench(args, local)["kernel"]}), flush=True)
        return
    if args.profile and args.profile_target in ("purity", "rk", "batched"):
        profile_case(args.profile_target, local)
        return
    eng = new_engine(1 if args.profile and args.profile_target == "split" else 0)
    if args.profile:
        eng.run_periods(1, is_obs=1)
        eng.close()
        return
    # transient: W untimed steps of P periods from |N,0>, then the window's start state
    for w in range(W):
        eng.run_periods(P, is_obs=1, dump_at=[P], dump_base=1 + w)
    snap = torch.empty(eng.checkpoint_size(), dtype=torch.uint8, pin_memory=True).numpy()
    snap = eng.checkpoint(out=snap)
    dev_ms_max, wall, clk, st0, st1, ens_plain, x_plain = timed_windows(eng, snap, ClockSampler(local))
    value = world * n * P * args.steps / (dev_ms_max * 1e-3)
    ms_per_step = dev_ms_max / args.steps
    ens_sum = ens_plain[-1]

    # roofline of the dominant kernel (step_kernel, grouped FP64 complex GEMM + fused epilogue)
    matvecs = st1["matvecs"] - st0["matvecs"]
    launches_step = st1["micro_steps"] - st0["micro_steps"]
    kern_ms = st1["step_kernel_ms"] - st0["step_kernel_ms"]
    flops = 8.0 * d * d * matvecs
    achieved = flops / (kern_ms * 1e-3) / 1e12
    peak_ffma, peak_dmma = q.measure_fp64_peak(local)
    peak = max(peak_ffma, peak_dmma)
    roofline = {"bound": "tensor", "pipe": "FP64 tensor core (mma.sync m8n8k4 f64; FP64 has no tcgen05 kind)",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_source": (f"measured live (qjx_measure_fp64_peak): FP64 tensor-core MMA chains {peak_dmma:.2f}, "
                                f"FFMA chains {peak_ffma:.2f} TFLOP/s; the larger is the peak"),
                "traffic": None, "kernel": kernel_name(d),
                "algorithmic_flops_per_launch": flops / max(launches_step, 1),
                "avg_launch_ms": kern_ms / max(launches_step, 1),
                "matvecs_per_traj_period": matvecs / (n * P * args.steps)}
    traffic_file = os.path.join(ROOT, "profiles", "step_kernel_traffic.json")
    if os.path.exists(traffic_file):
        with open(traffic_file) as f:
            tf = json.load(f)
        roofline["traffic"] = tf.get("bytes_per_launch")
        roofline["traffic_source"] = tf.get("source")

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": W, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(world, n, d, P, W),
        "wall_s": wall, "roofline": roofline, "clocks": clk,
        "gpu_launches": int(st1["launches"] - st0["launches"]),
        "ensemble_n1_minus_n2": ens_sum[0], "ensemble_n1_minus_n2_stderr": ens_sum[1],
        "matvecs_per_traj_period": matvecs / (n * P * args.steps),
    }
    if tuned:
        line["autotune"] = tuned

    # the split form and the other configurations' measurements: an error in one is reported in
    # its object and does not take the headline line with it
    def stage(fn, *a):
        try:
            return fn(*a)
        except Exception as ex:  # noqa: BLE001 -- recorded in the JSON line
            return {"error": f"{type(ex).__name__}: {ex}"}

    # split-precision form: same checkpoint, same windows
    if not args.no_split:
        line["split_form"] = stage(split_form, args, q, new_engine, timed_windows, snap, value, ens_plain, x_plain,
                                   eng, n, d, P, W, world)

    # e2e through the public C ABI with host buffers, copies inside the timed region
    if not args.no_e2e:
        barrier()
        t0 = time.perf_counter()
        for k in range(args.steps):
            slot = 1 + W + k
            eng.restore(snap)  # H2D: the window's start state from pinned host memory
            eng.run_periods(P, is_obs=1, dump_at=[P], dump_base=slot)
            ob = eng.observables(slot, 1)
            eng.states()
            allreduce([float(np.sum(N_BOSONS - 2.0 * ob["mean"][0])), float(n)])
        barrier()
        e2e_s = float(allreduce([time.perf_counter() - t0], "max")[0])
        line["e2e"] = {"value": world * n * P * args.steps / e2e_s, "unit": METRIC,
                       "h2d_bytes_per_step": int(snap.nbytes), "d2h_bytes_per_step": int(n * d * 16 + 5 * n * 8 + n * 16),
                       "path": "qjx_checkpoint_load (window start, pinned host buffer) + qjx_run_periods + "
                               "qjx_get_observables + qjx_get_states per step, same window as value"}
    if rank == 0 and not args.no_fbasis:
        line["fbasis"] = stage(fbasis_bench, args, local)
    if rank == 0 and world == 1 and not args.no_batch:  # single-GPU measurements
        line["batched"] = stage(batched_bench, args, local)
    if rank == 0 and world == 1 and not args.no_serve:
        line["serving"] = stage(serving_bench, args, local)
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample = CPU_TRAJ_PER_THREAD * threads
        rate, dt, mv = cpu_windows(M, sample, threads, W * P, P, 1)[0]
        line["cpu_baseline"] = {"value": rate, "unit": METRIC, "cores": threads, "kind": "port",
                                "sample": (f"trajectories 0..{sample - 1} x the same {P}-period window after the "
                                           f"same {W * P}-period transient ({dt:.1f} s timed), OpenMP over "
                                           f"trajectories, oracle/qjx_oracle.c"),
                                "matvecs_per_traj_period": mv}
    eng.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
