"""Continuous-batching request loop over serving engines (qjx_create_slots).

Each request is one dimer ensemble solve: N bosons (d = N + 1), n_traj trajectories, `periods`
periods, drive and dissipation parameters, a seed.  Requests are grouped by size class (d rounded
up to a power of two from 32, trajectories to 256, 1024, 4096 or 10240).  Each class runs in pools:
serving engines of a few slots of that class's size, each advancing all its loaded slots together,
one period per tick, in a thread of its own, so pools of different classes overlap on the device.
A pool keeps every admitted ensemble's trajectories resident on the device; between ticks it
retires the ensembles that reached their periods (observables and states read back) and loads
newly admitted ones into free slots.

Admission is by device memory: a request takes a free slot of a pool of its class; when there is
none, a new pool is created if its footprint fits the device's free memory (qjx_mem_info) minus a
reserve, closing idle pools to make room.  Otherwise the request waits, and requests of other
classes behind it are still admitted.

Operators are built ahead of admission on host threads, with the split tree on the GPU
(qjx_expm_tree: the host exponentials take about a minute at d = 1024, the GPU build
milliseconds).  A request's trajectories draw their own Philox streams (seed, tr_base), so its
result equals the same request solved alone with the same operators: identical states, jump
records and observables whatever it shares the device with (tests/test_serving_gpu.py).
"""
import collections
import concurrent.futures
import threading
import time

import numpy as np

from . import _native as N
from .engine import Engine

TWO_PI = 2.0 * 3.1415926535897932384626433832795
N_CLASSES = (256, 1024, 4096, 10240)


def dimer_ensemble(req, deep, device=0, gpu_build=True):
    """Operators of a request in the form Engine.slot_load takes: H, Hd, L on the host, the split
    tree on the GPU (build_dimer_gpu) or on the host (build_dimer)."""
    N_ = int(req["N"])
    E0, A, g = req.get("E0", 1.0), req.get("A", 1.5), req.get("g", 0.1)
    J, U, omega = req.get("J", 1.0), req.get("U", 0.5), req.get("omega", 1.0)
    if gpu_build:
        H, Hd, L, Ut = N.build_dimer_gpu(N_, J, U, E0, A, g, omega, deep, device)
    else:
        H, Hd, L, Ut = N.build_dimer(N_, J, U, E0, A, g, omega, deep)
    return dict(U=Ut, L=L, g=[1.0], HE=H + E0 * Hd, n_traj=int(req["n_traj"]), T=TWO_PI / omega,
                seed=int(req.get("seed", 0)), tr_base=int(req.get("tr_base", 0)))


def size_class(d, n_traj):
    """(d_cap, n_cap) of a request: d up to a power of two (at least 32), trajectories up to the
    next of 256, 1024, 4096, 10240."""
    d_cap = 32
    while d_cap < d:
        d_cap *= 2
    n_cap = next((c for c in N_CLASSES if c >= n_traj), None)
    if n_cap is None or d_cap > 1024:
        raise ValueError("request exceeds the largest size class (d <= 1024, 10240 trajectories)")
    return d_cap, n_cap


def pool_footprint(n_slots, d_cap, n_cap, deep, rec_cap=16, num_branches=2):
    """Device bytes of a serving engine of n_slots slots of (d_cap, n_cap) with one dump, no random
    observables and jump buffers of rec_cap records: matrices, two state slots, per-trajectory
    records and bucket lists (create_engine's allocations; checked against qjx_engine_bytes)."""
    md, kp = 8 * ((d_cap + 7) // 8), (d_cap + 1) & ~1
    ge = num_branches * deep + 2
    n, G = n_slots * n_cap, n_slots * ge
    mats = G * kp * md * 16
    psi = 2 * n * md * 16
    per_traj = 144 + 8 + 6 * 8 + 16 + 8 * d_cap + rec_cap * 28 + 1
    lists = 2 * G * n_cap * 4
    return mats + psi + n * per_traj + lists + 12 * G * 4 + (1 << 20)


class _Pool:
    """A serving engine of one size class and the thread that ticks it."""

    def __init__(self, server, d_cap, n_cap, n_slots):
        self.server = server
        self.d_cap, self.n_cap = d_cap, n_cap
        self.eng = Engine.slots(n_slots, d_cap, n_cap, deep=server.deep, max_dumps=1, rec_cap=16, device=server.device)
        self.bytes = self.eng.device_bytes()
        self.slots = [None] * n_slots  # request per slot (loaded, or waiting to load)
        self.loading = collections.deque()
        self.device_ms, self.ticks = 0.0, 0
        self.idle_since = time.perf_counter()
        self.closed = False
        self.error = None
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def free_slot(self):
        return next((i for i, r in enumerate(self.slots) if r is None), None)

    def active(self):
        return any(r is not None for r in self.slots)

    def _run(self):
        try:
            self._loop()
        except Exception as e:  # reported by Server.run
            with self.server.cv:
                self.error = e
                self.server.cv.notify_all()

    def _loop(self):
        srv = self.server
        while True:
            with srv.cv:
                while not self.closed and not self.loading and not any(r is not None and r.get("loaded")
                                                                       for r in self.slots):
                    srv.cv.wait(0.05)
                if self.closed:
                    return
                loads = list(self.loading)
                self.loading.clear()
            for slot, req in loads:  # between ticks: operators, states and thresholds of new requests
                self.eng.slot_load(slot, req["ops"])
                req["ops"] = None
                req["t_admit"] = srv.now()
                req["loaded"] = True
            self.eng.run_periods(1, is_obs=1, dump_at=[1], dump_base=0)
            self.device_ms += self.eng.stats()["last_call_ms"]
            self.ticks += 1
            done = []
            for i, r in enumerate(self.slots):
                if r is not None and r.get("loaded"):
                    r["left"] -= 1
                    if r["left"] == 0:
                        done.append(i)
            if not done:
                continue
            obs = self.eng.observables(0, 1)
            psi = self.eng.states()[0]
            for i in done:
                r = self.slots[i]
                sl = slice(i * self.n_cap, i * self.n_cap + int(r["n_traj"]))
                d = int(r["N"]) + 1
                r["result"] = {"mean": obs["mean"][0, sl].copy(), "norm": obs["norm"][0, sl].copy(),
                               "energy": obs["energy"][0, sl].copy(), "psi": psi[sl, :d].copy(),
                               "n1_minus_n2": float(np.mean(int(r["N"]) - 2.0 * obs["mean"][0, sl]))}
                r["t_done"] = srv.now()
                self.eng.slot_release(i)
            with srv.cv:
                for i in done:
                    srv.results.append(self.slots[i])
                    self.slots[i] = None
                if not self.active():
                    self.idle_since = time.perf_counter()
                srv.cv.notify_all()

    def close(self):
        with self.server.cv:
            self.closed = True
            self.server.cv.notify_all()
        self.thread.join()
        self.eng.close()


class Server:
    def __init__(self, deep=16, device=0, reserve_bytes=4 << 30, slots_per_pool=8, build_threads=4, gpu_build=True,
                 max_pools=16):
        self.deep, self.device = deep, device
        self.reserve = reserve_bytes
        self.slots_per_pool = slots_per_pool
        self.max_pools = max_pools
        self.gpu_build = gpu_build
        self.pools = []
        self.queue = collections.deque()
        self.results = []
        self.cv = threading.Condition()
        self.builder = concurrent.futures.ThreadPoolExecutor(max_workers=build_threads)
        self.t0 = time.perf_counter()
        self.pools_created = 0
        self.retired_device_ms = 0.0
        self.retired_ticks = 0
        self.peak_bytes = 0

    def now(self):
        return time.perf_counter() - self.t0

    @property
    def device_ms(self):
        return self.retired_device_ms + sum(p.device_ms for p in self.pools)

    @property
    def ticks(self):
        return self.retired_ticks + sum(p.ticks for p in self.pools)

    def submit(self, req):
        """Queue a request (dict: N, n_traj, periods, optional E0, A, g, J, U, omega, seed, tr_base)."""
        req = dict(req)
        req["cls"] = size_class(int(req["N"]) + 1, int(req["n_traj"]))
        req["t_submit"] = self.now()
        req["left"] = int(req["periods"])
        req["ops"] = self.builder.submit(dimer_ensemble, req, self.deep, self.device, self.gpu_build)
        self.queue.append(req)

    def busy(self):
        with self.cv:
            return bool(self.queue) or any(p.active() for p in self.pools)

    def _new_pool(self, cls):
        """A pool of class cls if its footprint fits the free device memory minus the reserve
        (closing idle pools to make room), else None."""
        need = pool_footprint(self.slots_per_pool, cls[0], cls[1], self.deep)
        free = N.mem_info(self.device)[0]
        if need + self.reserve > free:
            with self.cv:
                idle = sorted((p for p in self.pools if not p.active() and not p.loading), key=lambda p: p.idle_since)
            for p in idle:
                self._close_pool(p)
                free = N.mem_info(self.device)[0]
                if need + self.reserve <= free:
                    break
        if need + self.reserve > free or len(self.pools) >= self.max_pools:
            return None
        pool = _Pool(self, cls[0], cls[1], self.slots_per_pool)
        with self.cv:
            self.pools.append(pool)
        self.pools_created += 1
        self.peak_bytes = max(self.peak_bytes, sum(p.bytes for p in self.pools))
        return pool

    def _close_pool(self, p):
        with self.cv:
            self.pools.remove(p)
        self.retired_device_ms += p.device_ms
        self.retired_ticks += p.ticks
        p.close()

    def _admit(self):
        """First come first served per class: each queued request whose operators are built takes a
        free slot of a pool of its class, or of a new pool that fits the device memory."""
        waiting = collections.deque()
        while self.queue:
            req = self.queue.popleft()
            if not req["ops"].done():
                waiting.append(req)
                continue
            with self.cv:
                pool = next((p for p in self.pools if (p.d_cap, p.n_cap) == req["cls"] and p.free_slot() is not None),
                            None)
            if pool is None:
                pool = self._new_pool(req["cls"])
            if pool is None:
                waiting.append(req)
                continue
            req["ops"] = req["ops"].result()
            with self.cv:
                slot = pool.free_slot()
                pool.slots[slot] = req
                pool.loading.append((slot, req))
                self.cv.notify_all()
        self.queue = waiting

    def run(self, arrivals):
        """Serve (arrival_time_s, request) pairs in arrival order on the wall clock until all are done.
        On an error the pools are closed (their threads joined) before it propagates."""
        arrivals = sorted(arrivals, key=lambda x: x[0])
        k = 0
        try:
            while k < len(arrivals) or self.busy():
                while k < len(arrivals) and arrivals[k][0] <= self.now():
                    self.submit(arrivals[k][1])
                    k += 1
                self._admit()
                with self.cv:
                    err = next((p.error for p in self.pools if p.error is not None), None)
                    if err is not None:
                        raise err
                    self.cv.wait(0.005)
        except BaseException:
            self.close()
            raise
        return list(self.results)

    def close(self):
        for p in list(self.pools):
            self._close_pool(p)
        self.builder.shutdown(wait=True)
