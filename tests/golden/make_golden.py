"""Generates tests/golden/qj_dim11_seed42.npz from the CPU oracle (run from the repo root:
python tests/golden/make_golden.py).  The fixture freezes a small QJ ensemble: dimer N = 10,
12 trajectories, 1 transient and 3 observation periods, Philox seed 42, one dump per period."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle_py as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "qj_dim11_seed42.npz")
N, n, tp, periods, seed, deep = 10, 12, 1, 3, 42, 16


def compute():
    H, Hd, L, K0, K1 = O.dimer_operators(N, 1.0, 0.5, 1.0, 1.5, 0.1)
    T = 2.0 * 3.1415926535897932384626433832795
    U = np.stack([O.split_tree(K0, T, deep), O.split_tree(K1, T, deep)])
    ens = O.Ensemble(U, L, [1.0], H + Hd, None, T, n, seed=seed, record=2)
    ens.init(0, 0)
    assert ens.run_periods(tp, is_obs=0) == 0
    ens.t[:] = 0.0
    obs = [ens.observables(is_start=True)]
    for _ in range(periods):
        assert ens.run_periods(1) == 0
        obs.append(ens.observables())
    out = {"psi": ens.phi.copy(), "t": ens.t.copy(), "eta": ens.eta.copy(), "jumps_counts": ens.jumps_counts.copy()}
    for k in ("norm", "mean", "dispersion", "m2", "energy"):
        out["obs_" + k] = np.stack([o[k] for o in obs])
    counts = ens.n_rec.copy()
    out["rec_counts"] = counts
    out["jump_times"] = np.concatenate([ens.jumps(tr)[0] for tr in range(n)])
    out["diss_types"] = np.concatenate([ens.jumps(tr)[1] for tr in range(n)])
    out["jump_norms"] = np.concatenate([ens.jumps(tr)[2] for tr in range(n)])
    out["jump_etas"] = np.concatenate([ens.jumps(tr)[3] for tr in range(n)])
    return out


if __name__ == "__main__":
    np.savez_compressed(OUT, **compute())
    print("wrote", OUT)
