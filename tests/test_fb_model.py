"""The library's f-basis Liouvillian builder (qjx_fb_build_dimer, banded projection) against the
oracle's dense projection (oracle/fbasis_oracle.c): same sparsity pattern, same values."""
import numpy as np
import pytest

from oracle import oracle_py as O


@pytest.mark.parametrize("N,J,U,E,g", [(4, 1.0, 0.5, 1.0, 2.0), (12, 1.0, 0.5, 1.0, 0.1), (25, 0.7, 1.3, -0.4, 0.3)])
def test_builder_matches_oracle_projection(N, J, U, E, g):
    from os_d_b200 import _native as Nt

    (gr, gc, gv), (qr, qc, qv), ks = Nt.fb_build_dimer(N, J, U, E, g)
    Gs, Qs, Ks = O.fb_dense(N, J, U, E, g)
    G, Q = O.fb_csr(Gs), O.fb_csr(Qs)
    assert np.array_equal(gr, G.indptr) and np.array_equal(gc, G.indices)
    assert np.array_equal(qr, Q.indptr) and np.array_equal(qc, Q.indices)
    scale = np.abs(Gs).max()
    assert np.abs(gv - G.data).max() < 1e-13 * scale
    assert np.abs(qv - Q.data).max() < 1e-13 * np.abs(Qs).max()
    assert np.abs(ks - Ks).max() < 1e-13 * max(np.abs(Ks).max(), 1.0)


def test_builder_rejects_bad_sizes():
    from os_d_b200 import _native as Nt

    with pytest.raises(Nt.QjxError):
        Nt.fb_build_dimer(0, 1.0, 0.5, 1.0, 0.1)


@pytest.mark.parametrize("N,k", [(3, 0), (7, 2), (7, 7), (20, 11)])
def test_pure_state_vector_matches_init_rho(N, k):
    import os_d_b200 as q

    rho = np.zeros((N + 1, N + 1), complex)
    rho[k, k] = 1
    assert np.allclose(q.fbasis_pure_state(N, k), O.fb_x_from_rho(N, rho), atol=1e-15)
