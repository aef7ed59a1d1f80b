"""Known-answer tests that pin the CPU oracle (no GPU).

The reference cannot be built here (Intel MKL and Eigen are absent) and ships no golden
data, so the oracle is pinned to independent facts:
  * Philox4x32-10 known-answer vectors (Random123, Salmon et al. 2011)
  * Pade coefficients of Higham (2005) against the factorial formula, expm against scipy
  * the dimer operators against the reference's own MATLAB generator of the same
    matrices (qj_input/qj_input.m:46-95), restated here in numpy
  * the split tree: U_l = U_{l+1}^2, dt halving (qj_proc.cpp:15-24)
  * the recursion of one_period_branch (qj_proc.cpp:271-343) against a separate
    pure-Python restatement
  * the physics: the QJ ensemble against the exact dense Lindblad evolution
    (source/matlab/origin/dimer/sysLind.m:14-15) within statistical error
"""
from fractions import Fraction
from math import factorial

import numpy as np
import pytest
import scipy.linalg as sla

from oracle import oracle_py as O
from tests.helpers import T2PI, dimer_problem


def test_philox_known_answers():
    assert O.philox4x32_10([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert O.philox4x32_10([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert O.philox4x32_10([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_philox_uniforms_in_open_closed_interval():
    u = np.array([O.philox_uniform(42, tr, i) for tr in range(4) for i in range(500)])
    assert u.min() > 0.0 and u.max() <= 1.0
    assert abs(u.mean() - 0.5) < 0.03
    # draw i of trajectory tr is a pure function of (seed, tr, i)
    assert O.philox_uniform(7, 3, 11) == O.philox_uniform(7, 3, 11) != O.philox_uniform(7, 4, 11)


@pytest.mark.parametrize("m", [3, 5, 7, 9, 13])
def test_pade_coefficients_match_factorial_formula(m):
    table = {3: [120, 60, 12, 1], 5: [30240, 15120, 3360, 420, 30, 1],
             7: [17297280, 8648640, 1995840, 277200, 25200, 1512, 56, 1],
             9: [17643225600, 8821612800, 2075673600, 302702400, 30270240, 2162160, 110880, 3960, 90, 1],
             13: [64764752532480000, 32382376266240000, 7771770303897600, 1187353796428800, 129060195264000,
                  10559470521600, 670442572800, 33522128640, 1323241920, 40840800, 960960, 16380, 182, 1]}[m]
    c = [Fraction(factorial(2 * m - j) * factorial(m), factorial(2 * m) * factorial(j) * factorial(m - j))
         for j in range(m + 1)]
    assert [ci / c[m] for ci in c] == [Fraction(t) for t in table]


@pytest.mark.parametrize("scale", [1e-3, 0.05, 0.5, 1.5, 5.0, 40.0, 300.0])
def test_expm_matches_scipy(scale):
    rng = np.random.default_rng(int(scale * 1000))
    A = (rng.standard_normal((24, 24)) + 1j * rng.standard_normal((24, 24))) * scale / 24
    e1, e2 = O.expm(A), sla.expm(A)
    assert np.abs(e1 - e2).max() <= 1e-12 * max(1.0, np.abs(e2).max())


def test_expm_dimer_generator_matches_scipy():
    P = dimer_problem(60, deep=4)
    H, Hd, L, K0, K1 = O.dimer_operators(60, 1.0, 0.5, 1.0, 1.5, 0.1)
    for dt in (T2PI / 4, T2PI / 64, T2PI / 2 ** 17):
        e1, e2 = O.expm(K0 * dt), sla.expm(K0 * dt)
        assert np.abs(e1 - e2).max() <= 1e-11 * np.abs(e2).max()
    assert P["U"].shape == (2, 4, 61, 61)


def qj_input_operators(d, J, U, E, A, g):
    """numpy restatement of qj_input/qj_input.m:33-95 (d = matrix size)."""
    U, g = U / (d - 1), g / (d - 1)
    A1 = np.diag(np.arange(d, dtype=float))
    A2 = np.diag(d - 1 - np.arange(d, dtype=float))
    H2 = A2 - A1
    H1 = U * 2 * (A1 @ (A1 - np.eye(d)) + A2 @ (A2 - np.eye(d)))
    V = A1 - A2
    for i in range(1, d):  # 1-based i of the .m file
        s = np.sqrt((d - i) * i)
        H1[i, i - 1] -= J * s
        H1[i - 1, i] -= J * s
        V[i, i - 1] -= s
        V[i - 1, i] += s
    ham = H1 + E * H2
    Heff = H1 - 0.5j * (g * V.conj().T @ V)
    return ham, H1, H2, V, -1j * (Heff + (E + A) * H2), -1j * (Heff + (E - A) * H2)


@pytest.mark.parametrize("N,J,U,E,A,g", [(10, 1.0, 0.5, 1.0, 1.5, 0.1), (37, -0.7, 0.13, 0.0, 3.4, 0.02)])
def test_operators_match_reference_matlab_generator(N, J, U, E, A, g):
    H, Hd, L, K0, K1 = O.dimer_operators(N, J, U, E, A, g)
    ham, H1, H2, V, K0m, K1m = qj_input_operators(N + 1, J, U, E, A, g)
    assert np.allclose(H, H1, atol=1e-13, rtol=0)
    assert np.array_equal(Hd.real, H2) and not Hd.imag.any()
    assert np.allclose(L, V, atol=1e-13, rtol=0)
    assert np.allclose(K0, K0m, atol=1e-12, rtol=0) and np.allclose(K1, K1m, atol=1e-12, rtol=0)
    # closed forms of the reference (newdel.cpp:484-496, 1486-1496)
    k = np.arange(N + 1)
    assert np.allclose(np.diag(H).real, 2 * (U / N) * (k * (k - 1) + (N - k) * (N - k - 1)))
    assert np.array_equal(np.diag(L).real, 2.0 * k - N)


def test_split_tree_is_consistent():
    P = dimer_problem(30, deep=8)
    U = P["U"]
    for b in range(2):
        for lvl in range(7):
            assert np.abs(U[b, lvl + 1] @ U[b, lvl + 1] - U[b, lvl]).max() < 1e-12 * np.abs(U[b, lvl]).max()
    # the non-Hermitian part only damps: singular values <= 1
    assert np.linalg.svd(U[0, 0], compute_uv=False).max() <= 1.0 + 1e-12


def test_matvec_contract_equals_numpy_to_rounding():
    rng = np.random.default_rng(1)
    M = rng.standard_normal((57, 57)) + 1j * rng.standard_normal((57, 57))
    x = rng.standard_normal(57) + 1j * rng.standard_normal(57)
    assert np.allclose(O.matvec(M, x), M @ x, rtol=1e-14, atol=1e-13)
    assert abs(O.norm_square(x) - np.vdot(x, x).real) < 1e-13 * np.vdot(x, x).real


@pytest.mark.parametrize("dump_type,dump_num,nobs", [(0, 4, 20), (0, 3, 10), (1, 5, 1000), (1, 3, 50)])
def test_dump_periods(dump_type, dump_num, nobs):
    got = list(O.dump_periods(dump_type, dump_num, nobs))
    if dump_type == 0:
        exp = [0] + [(i + 1) * (nobs // dump_num) for i in range(dump_num)]
    else:
        exp = [0]
        per = dump_num / np.log10(nobs)
        for i in range(dump_num + 1):
            cur = int(10 ** 0 * 10 ** ((1 / per) * i))
            exp.append(cur if cur > exp[-1] else exp[-1] + 1)
    assert got == exp


# ---------------------------------------------------------------- independent recursion
def python_qj(U, L, T, n_periods, etas_draws, psi0):
    """Literal restatement of one_period_branch / recovery (qj_proc.cpp:271-343,
    experiment.cpp:1273-1382) in plain numpy, fed the same uniforms."""
    deep = U.shape[1]
    dts = []
    dt = T * 0.5
    for _ in range(deep):
        dt *= 0.5
        dts.append(dt)
    st = {"psi": psi0.copy(), "t": 0.0, "pos": 0, "jumps": []}

    def draw():
        u = etas_draws[st["pos"]]
        st["pos"] += 1
        return u

    st["eta"] = draw()

    def branch(b, lvl):
        for _ in range(2):
            aux = U[b, lvl] @ st["psi"]
            nrm = np.vdot(aux, aux).real
            crossed = not (nrm > st["eta"])
            if lvl == deep - 1:
                if crossed:
                    st["jumps"].append(st["t"] + dts[lvl])
                    aux = aux / np.sqrt(nrm)
                    draw()  # channel choice (one channel)
                    r = L @ aux
                    aux = r / np.sqrt(np.vdot(r, r).real)
                    st["eta"] = draw()
                st["psi"] = aux
            else:
                if crossed:
                    branch(b, lvl + 1)
                    st["t"] -= dts[lvl]
                else:
                    st["psi"] = aux
            st["t"] += dts[lvl]

    for _ in range(n_periods):
        for b in range(2):
            branch(b, 0)
    return st


def test_oracle_recursion_matches_independent_restatement():
    N, n, periods = 6, 6, 3
    P = dimer_problem(N, deep=10)
    rng = np.random.default_rng(11)
    lens = np.full(n, 4000)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    u = rng.random(off[-1])
    u[u == 0] = 0.5
    ens = O.Ensemble(P["U"], P["L"], [1.0], P["HE"], None, P["T"], n, record=2, rng_kind=1, inj_u=u, inj_off=off)
    ens.init(0, 0)
    assert ens.run_periods(periods) == 0
    psi0 = np.zeros(N + 1, complex)
    psi0[0] = 1
    for tr in range(n):
        ref = python_qj(P["U"], P["L"], P["T"], periods, u[off[tr]:off[tr + 1]], psi0)
        t_o = ens.jumps(tr)[0]
        assert len(t_o) == len(ref["jumps"]) > 0
        assert np.allclose(t_o, ref["jumps"], rtol=0, atol=1e-12)
        assert np.allclose(ens.phi[tr], ref["psi"], atol=1e-10)
        assert ens.rng_pos[tr] == ref["pos"]


def test_weak_dissipation_has_no_jumps_and_keeps_norm():
    H, Hd, L, K0, K1 = O.dimer_operators(12, 1.0, 0.5, 1.0, 1.5, 1e-7)
    U = np.stack([O.split_tree(K0, T2PI, 16), O.split_tree(K1, T2PI, 16)])
    ens = O.Ensemble(U, L, [1.0], H + Hd, None, T2PI, 16, seed=3, record=1)
    ens.init(0, 0)
    ens.eta[:] = 0.5  # a threshold far below the norm
    assert ens.run_periods(3) == 0
    assert ens.jumps_counts.sum() == 0
    nrm = (np.abs(ens.phi) ** 2).sum(axis=1)
    assert np.all(nrm <= 1.0) and np.all(nrm > 1 - 1e-4)


# ---------------------------------------------------------------- physics against Lindblad
def lindblad_period_map(H, Hd, L, E, A, g, N, T):
    """Exact one-period map of dρ/dt = -i[H + E(t) Hd, ρ] + γ (LρL† - ½{L†L, ρ}), γ = g/N,
    E(t) = E + A on the first half period and E - A on the second (row-major vec)."""
    d = H.shape[0]
    I = np.eye(d)
    gam = g / N
    LdL = L.conj().T @ L

    def liou(Ht):
        return (-1j * (np.kron(Ht, I) - np.kron(I, Ht.T))
                + gam * (np.kron(L, L.conj()) - 0.5 * np.kron(LdL, I) - 0.5 * np.kron(I, LdL.T)))

    M0 = sla.expm(liou(H + (E + A) * Hd) * (T / 2))
    M1 = sla.expm(liou(H + (E - A) * Hd) * (T / 2))
    return M1 @ M0


def test_qj_ensemble_matches_lindblad_populations():
    N, n, periods = 4, 3000, 4
    E, A, g = 1.0, 1.5, 2.0
    H, Hd, L, K0, K1 = O.dimer_operators(N, 1.0, 0.5, E, A, g)
    U = np.stack([O.split_tree(K0, T2PI, 16), O.split_tree(K1, T2PI, 16)])
    ens = O.Ensemble(U, L, [1.0], H + E * Hd, None, T2PI, n, seed=5, record=1)
    ens.init(0, 0)
    Mp = lindblad_period_map(H, Hd, L, E, A, g, N, T2PI)
    rho = np.zeros((N + 1, N + 1), complex)
    rho[0, 0] = 1
    vec = rho.reshape(-1)
    for _ in range(periods):
        assert ens.run_periods(1) == 0
        vec = Mp @ vec
        pops_l = np.real(np.diag(vec.reshape(N + 1, N + 1)))
        adr = ens.observables(want_adr=True)["adr"]
        pops_q = adr.mean(axis=0)
        err = adr.std(axis=0) / np.sqrt(n)
        assert np.all(np.abs(pops_q - pops_l) < 4.5 * err + 1e-3), (pops_q, pops_l)
    assert ens.jumps_counts.sum() > n  # the test exercises jumps
