"""The allocation-free f-basis RK4 entry point (qjx_fb_rk4_noalloc) against the allocating one.

qjx_fb_rk4_noalloc is for callers that cannot let this library allocate GPU memory (a host
program that owns all device buffers through its own pool, or a solver loop that must not
pay cudaMalloc's device-wide synchronisation mid-run): the caller passes device buffers for
the inputs and the state, and the RK4 stage vectors live in a fixed static device array.
This file is collected last so a stop at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle_py as O
from tests.helpers import T2PI

pytestmark = pytest.mark.gpu


def _device_arrays(torch, *arrays):
    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrays]


def test_noalloc_rk4_matches_allocating_entry_point_on_two_calls():
    import torch

    import os_d_b200 as q
    from os_d_b200 import _native as N

    Nb, steps = 20, 300
    Gs, Qs, Ks = O.fb_dense(Nb, 1.0, 0.5, 1.0, 0.1)
    Gc, Qc = O.fb_csr(Gs), O.fb_csr(Qs)
    rho0 = np.zeros((Nb + 1, Nb + 1), complex)
    rho0[0, 0] = 1
    x0 = O.fb_x_from_rho(Nb, rho0)
    n = x0.size

    # reference values: the allocating entry point, after one and after two periods
    fb = q.FBasis(Gc, Qc, Ks, x0, 1.5, drv_type=0, T=T2PI, num_steps=steps)
    fb.run(0, 1)
    x_one, _ = fb.get()
    fb.run(1, 1)
    x_two, _ = fb.get()
    fb.close()

    # caller-owned device buffers (the caller may allocate; the entry point does not)
    gr, gc, gv, qr, qc, qv, ks, x = _device_arrays(
        torch, Gc.indptr.astype(np.int32), Gc.indices.astype(np.int32), Gc.data, Qc.indptr.astype(np.int32),
        Qc.indices.astype(np.int32), Qc.data, Ks, x0)
    stream = torch.cuda.current_stream().cuda_stream
    lib = N.lib()

    def call(period0):
        st = lib.qjx_fb_rk4_noalloc(n, gr.data_ptr(), gc.data_ptr(), gv.data_ptr(), qr.data_ptr(), qc.data_ptr(),
                                    qv.data_ptr(), ks.data_ptr(), x.data_ptr(), 1.5, 1.0, 0.0, 0, T2PI, steps,
                                    period0, 1, torch.cuda.current_device(), C.c_void_p(stream))
        assert st == 0, lib.qjx_status_string(st)
        torch.cuda.synchronize()
        return x.cpu().numpy()

    assert np.array_equal(call(0), x_one)   # first call (also the per-device set-up)
    assert np.array_equal(call(1), x_two)   # second call reuses the shared static array


def test_noalloc_rejects_sizes_beyond_its_static_array():
    import torch

    from os_d_b200 import _native as N

    lib = N.lib()
    big = 65536 + 1
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    st = lib.qjx_fb_rk4_noalloc(big, p, p, p, p, p, p, p, p, 1.0, 1.0, 0.0, 0, T2PI, 10, 0, 1,
                                torch.cuda.current_device(), None)
    assert lib.qjx_status_string(st) == b"unsupported configuration"


@pytest.mark.parametrize("N,steps,T", [(100, 50, 0.2), (199, 6, 0.012)])
def test_noalloc_rk4_large_systems_match_oracle_on_two_calls(N, steps, T):
    """Sizes far beyond one wave of resident blocks (n = 10,200 and 39,999): every row of a stage
    reads other rows' stage arguments, so the stage buffers must not be overwritten within a
    launch.  Two calls in a row (periods 15 and 16; at N = 100 the drive changes sign inside the
    first, at t = pi) equal the oracle's RK4 bit for bit."""
    import torch

    import os_d_b200 as q
    from os_d_b200 import _native as Nt

    (grh, gch, gvh), (qrh, qch, qvh), ksh = Nt.fb_build_dimer(N, 1.0, 0.5, 1.0, 0.1)
    import scipy.sparse as sp

    n = (N + 1) ** 2 - 1
    assert n <= 65536
    Gc, Qc = sp.csr_matrix((gvh, gch, grh), shape=(n, n)), sp.csr_matrix((qvh, qch, qrh), shape=(n, n))
    x0 = q.fbasis_pure_state(N, 0)
    gr, gc, gv, qr, qc, qv, ks, x = _device_arrays(torch, grh, gch, gvh, qrh, qch, qvh, ksh, x0)
    stream = torch.cuda.current_stream().cuda_stream
    lib = Nt.lib()
    x_ref = x0
    for period in (15, 16):
        st = lib.qjx_fb_rk4_noalloc(n, gr.data_ptr(), gc.data_ptr(), gv.data_ptr(), qr.data_ptr(), qc.data_ptr(),
                                    qv.data_ptr(), ks.data_ptr(), x.data_ptr(), 1.5, 1.0, 0.0, 0, T, steps,
                                    period, 1, torch.cuda.current_device(), C.c_void_p(stream))
        assert st == 0, lib.qjx_status_string(st)
        torch.cuda.synchronize()
        x_ref = O.fb_rk4(Gc, Qc, ksh, x_ref, 1.5, drv_type=0, T=T, num_steps=steps, period0=period, n_periods=1)
        assert np.array_equal(x.cpu().numpy(), x_ref)
    assert np.abs(x_ref - x0).max() > 1e-8
