"""Host logic of the serving loop (os_d_b200.serve) on the CPU: size classes, pool creation
against free memory, admission, per-request slots and results, and the error path, with a
stand-in for the serving engine (the operators are built by the library's host builder)."""
import threading

import numpy as np
import pytest

from os_d_b200 import serve


class FakeSlots:
    """The serving engine's interface: each tick advances every loaded slot by one period and
    writes the slot's index into its trajectories' 'mean' so results can be traced to slots."""

    created = 0
    fail_on = None  # the creation number that raises (1-based), or None

    def __init__(self, n_slots, d_cap, n_cap):
        FakeSlots.created += 1
        if FakeSlots.fail_on == FakeSlots.created:
            raise RuntimeError("qjx_create_slots failed (7): CUDA error")
        self.n_slots, self.d_cap, self.n_cap = n_slots, d_cap, n_cap
        self.loaded = [None] * n_slots
        self.periods = np.zeros(n_slots, int)

    @classmethod
    def slots(cls, n_slots, d_cap, n_cap, **kw):
        return cls(n_slots, d_cap, n_cap)

    def device_bytes(self):
        return serve.pool_footprint(self.n_slots, self.d_cap, self.n_cap, 16)

    def slot_load(self, slot, ens):
        assert ens["U"].shape[-1] <= self.d_cap and ens["n_traj"] <= self.n_cap
        self.loaded[slot] = ens
        self.periods[slot] = 0

    def slot_release(self, slot):
        self.loaded[slot] = None

    def run_periods(self, k, **kw):
        for i, e in enumerate(self.loaded):
            if e is not None:
                self.periods[i] += k

    def stats(self):
        return {"last_call_ms": 1.0}

    def observables(self, dump, n):
        n_all = self.n_slots * self.n_cap
        mean = np.repeat(np.arange(self.n_slots, dtype=float), self.n_cap)[None, :]
        return {"mean": mean, "norm": np.ones((1, n_all)), "energy": np.zeros((1, n_all))}

    def states(self):
        return (np.zeros((self.n_slots * self.n_cap, self.d_cap), complex),)

    def close(self):
        pass


@pytest.fixture
def fake(monkeypatch):
    FakeSlots.created, FakeSlots.fail_on = 0, None
    monkeypatch.setattr(serve, "Engine", FakeSlots)
    monkeypatch.setattr(serve.N, "mem_info", lambda device=0: (1 << 40, 1 << 40))
    return FakeSlots


def requests(k, rng):
    out = []
    for i in range(k):
        out.append((0.001 * i, dict(N=int(rng.integers(8, 70)), n_traj=int(rng.integers(5, 300)),
                                    periods=int(rng.integers(1, 4)), E0=1.0, g=0.1, seed=i, tr_base=1000 * i)))
    return out


def test_size_classes():
    assert serve.size_class(21, 100) == (32, 256)
    assert serve.size_class(33, 257) == (64, 1024)
    assert serve.size_class(1024, 10240) == (1024, 10240)
    with pytest.raises(ValueError):
        serve.size_class(1025, 10)
    with pytest.raises(ValueError):
        serve.size_class(100, 10241)


def test_every_request_is_served_in_its_class_and_slot(fake):
    arrivals = requests(12, np.random.default_rng(1))
    srv = serve.Server(deep=4, slots_per_pool=2, reserve_bytes=0, gpu_build=False)
    res = srv.run(arrivals)
    created = srv.pools_created
    srv.close()
    assert len(res) == 12 and created >= 2
    seen = {(r["seed"], r["tr_base"]) for r in res}
    assert seen == {(r["seed"], r["tr_base"]) for _, r in arrivals}
    for r in res:
        assert r["t_done"] >= r["t_admit"] >= r["t_submit"]
        assert r["left"] == 0
        d_cap, n_cap = r["cls"]
        assert int(r["N"]) + 1 <= d_cap and int(r["n_traj"]) <= n_cap
        # the result is the request's own slice of its slot: one value, the slot's index
        mean = r["result"]["mean"]
        assert mean.shape == (int(r["n_traj"]),) and np.all(mean == mean[0])
        assert r["result"]["psi"].shape == (int(r["n_traj"]), int(r["N"]) + 1)


def test_a_failing_pool_creation_raises_and_leaves_no_pool_thread(fake):
    fake.fail_on = 2
    before = threading.active_count()
    arrivals = [(0.0, dict(N=10, n_traj=20, periods=2, seed=1)), (0.0, dict(N=60, n_traj=20, periods=2, seed=2)),
                (0.0, dict(N=200, n_traj=20, periods=2, seed=3))]
    srv = serve.Server(deep=4, slots_per_pool=2, reserve_bytes=0, gpu_build=False)
    with pytest.raises(RuntimeError, match="qjx_create_slots"):
        srv.run(arrivals)
    assert not srv.pools
    assert threading.active_count() <= before
