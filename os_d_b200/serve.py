"""Continuous-batching request loop over a serving engine (qjx_create_slots).

Each request is one dimer ensemble solve: N bosons (d = N + 1), n_traj trajectories, `periods`
periods, drive and dissipation parameters, a seed.  The loop keeps every admitted ensemble's
trajectories resident on the device in a slot of one engine and advances all loaded slots
together, one period per tick (the engine's grouped micro-step launches).  Between ticks it
retires the ensembles that reached their periods (observables and states read from the device)
and admits queued requests, first come first served, while a slot is free and the HBM footprint
of the admitted ensembles stays within the budget.  Operators are built on host threads ahead of
admission, so building overlaps the device work.

A request's trajectories draw their own Philox streams (seed, tr_base), so its result is the one
it would get alone: identical states, jump records and observables whatever it shares the device
with (tests/test_serving_gpu.py).
"""
import collections
import concurrent.futures
import time

import numpy as np

from . import _native as N
from .engine import Engine

TWO_PI = 2.0 * 3.1415926535897932384626433832795


def dimer_ensemble(req, deep):
    """Operators of a request (qjx_build_dimer), in the form Engine.slot_load takes."""
    N_ = int(req["N"])
    E0, A, g = req.get("E0", 1.0), req.get("A", 1.5), req.get("g", 0.1)
    J, U, omega = req.get("J", 1.0), req.get("U", 0.5), req.get("omega", 1.0)
    H, Hd, L, Ut = N.build_dimer(N_, J, U, E0, A, g, omega, deep)
    return dict(U=Ut, L=L, g=[1.0], HE=H + E0 * Hd, n_traj=int(req["n_traj"]), T=TWO_PI / omega,
                seed=int(req.get("seed", 0)), tr_base=int(req.get("tr_base", 0)))


def footprint(d, n_traj, deep, num_branches=2):
    """Device bytes of one admitted ensemble: two state slots, the split tree, L and the energy
    operator (complex FP64, rows padded to 8)."""
    md = 8 * ((d + 7) // 8)
    return 2 * n_traj * md * 16 + (num_branches * deep + 2) * ((d + 1) & ~1) * md * 16


class Server:
    def __init__(self, n_slots, d_cap, n_cap, deep=16, hbm_budget=None, device=0, build_threads=4):
        self.eng = Engine.slots(n_slots, d_cap, n_cap, deep=deep, max_dumps=1, device=device)
        self.deep, self.d_cap, self.n_cap = deep, d_cap, n_cap
        self.budget = hbm_budget
        self.used = 0
        self.slots = [None] * n_slots
        self.queue = collections.deque()
        self.results = []
        self.pool = concurrent.futures.ThreadPoolExecutor(max_workers=build_threads)
        self.t0 = time.perf_counter()
        self.device_ms = 0.0
        self.ticks = 0

    def now(self):
        return time.perf_counter() - self.t0

    def submit(self, req):
        """Queue a request (dict: N, n_traj, periods, optional E0, A, g, J, U, omega, seed, tr_base)."""
        if int(req["N"]) + 1 > self.d_cap or int(req["n_traj"]) > self.n_cap:
            raise ValueError("request exceeds the slot capacity")
        req = dict(req)
        req["t_submit"] = self.now()
        req["ops"] = self.pool.submit(dimer_ensemble, req, self.deep)
        req["bytes"] = footprint(int(req["N"]) + 1, int(req["n_traj"]), self.deep)
        self.queue.append(req)

    def busy(self):
        return bool(self.queue) or any(s is not None for s in self.slots)

    def _admit(self):
        while self.queue:
            req = self.queue[0]
            free = [i for i, s in enumerate(self.slots) if s is None]
            if not free or (self.budget is not None and self.used + req["bytes"] > self.budget):
                return
            self.queue.popleft()
            slot = free[0]
            self.eng.slot_load(slot, req["ops"].result())
            req["ops"] = None
            req["t_admit"] = self.now()
            req["left"] = int(req["periods"])
            self.used += req["bytes"]
            self.slots[slot] = req

    def _retire(self):
        done = [i for i, r in enumerate(self.slots) if r is not None and r["left"] == 0]
        if not done:
            return
        obs = self.eng.observables(0, 1)
        psi = self.eng.states()[0]
        for i in done:
            r = self.slots[i]
            sl = slice(i * self.n_cap, i * self.n_cap + int(r["n_traj"]))
            d = int(r["N"]) + 1
            r["result"] = {"mean": obs["mean"][0, sl].copy(), "norm": obs["norm"][0, sl].copy(),
                           "energy": obs["energy"][0, sl].copy(), "psi": psi[sl, :d].copy(),
                           "n1_minus_n2": float(np.mean(int(r["N"]) - 2.0 * obs["mean"][0, sl]))}
            r["t_done"] = self.now()
            self.eng.slot_release(i)
            self.used -= r["bytes"]
            self.slots[i] = None
            self.results.append(r)

    def tick(self):
        """Admit, advance every loaded slot by one period (observables at its end), retire."""
        self._admit()
        if not any(s is not None for s in self.slots):
            return False
        self.eng.run_periods(1, is_obs=1, dump_at=[1], dump_base=0)
        self.device_ms += self.eng.stats()["last_call_ms"]
        self.ticks += 1
        for r in self.slots:
            if r is not None:
                r["left"] -= 1
        self._retire()
        return True

    def run(self, arrivals):
        """Serve (arrival_time_s, request) pairs in arrival order on the wall clock until all are done."""
        arrivals = sorted(arrivals, key=lambda x: x[0])
        k = 0
        while k < len(arrivals) or self.busy():
            while k < len(arrivals) and arrivals[k][0] <= self.now():
                self.submit(arrivals[k][1])
                k += 1
            if not self.tick() and k < len(arrivals):
                time.sleep(max(0.0, min(0.01, arrivals[k][0] - self.now())))
        return self.results

    def close(self):
        self.pool.shutdown(wait=True)
        self.eng.close()
