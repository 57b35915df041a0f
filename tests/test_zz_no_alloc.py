"""bec_moments_device_noalloc: moments of states in the caller's device memory,
computed without any device allocation (for callers that cannot let the
library call cudaMalloc: hosts that own all device memory through their own
pool, and loops that must never block on an allocation).

Checked through the C ABI against an FP64 NumPy sum of the same array and
against bec_moments_now of a context holding the same states, on calls in a
row with different inputs and sizes: a large call whose grid-stride first
stage is clamped to the 1024 partial sums of the scratch array, then smaller
calls that must not pick up the partial sums the large call left behind.
After a warm-up call, the calls leave the device's free memory unchanged.
This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from bec_b200._abi import BEC_ERR_INVALID_ARG, BEC_OK
from bec_b200.configs import rb87_params
from bec_b200.engine import BEC_PATH_FP64_PLAIN, Engine, lib

pytestmark = pytest.mark.gpu

TOL = 1e-10   # the FP64 parity bound of the GPU tests


def _states(grid, ne, seed):
    p = rb87_params(N=30000, grid=grid, ne=ne, noise=True)
    rng = np.random.default_rng(seed)
    with Engine([p], path=BEC_PATH_FP64_PLAIN) as eng:
        d = eng.derived[0]
        psi = (rng.standard_normal((ne, 2, d.cells)) + 1j * rng.standard_normal((ne, 2, d.cells))) * 3.0
        eng.init_group(0, np.zeros(d.cells))
        for t in range(ne):
            eng.set_state(0, t, psi[t])
        expect = eng.moments()[0]
        return psi, d.cells, d.dV, expect


def _noalloc(psi, cells, ne, dV):
    import torch
    dev = torch.from_numpy(np.ascontiguousarray(psi).view(np.float64).reshape(-1).copy()).cuda()
    out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = lib().bec_moments_device_noalloc(C.c_void_p(dev.data_ptr()), cells, ne, dV, C.c_void_p(out.data_ptr()),
                                          None)
    torch.cuda.synchronize()
    return st, out.cpu().numpy()


def _numpy_moments(psi, dV):
    a, b = psi[:, 0], psi[:, 1]
    s = (np.conj(a) * b).sum()
    return np.array([(np.abs(a) ** 2).sum(), (np.abs(b) ** 2).sum(), s.real, s.imag]) * dV


def test_noalloc_moments_match_context_moments_twice():
    cases = [((16, 16, 128), 3, 1), ((8, 8, 64), 2, 2)]
    for grid, ne, seed in cases:
        psi, cells, dV, expect = _states(grid, ne, seed)
        st, got = _noalloc(psi, cells, ne, dV)
        assert st == BEC_OK
        np.testing.assert_allclose(got, expect[1:], rtol=TOL, atol=TOL * np.abs(expect[1:3]).max())
        ref = _numpy_moments(psi, dV)
        np.testing.assert_allclose(got, ref, rtol=TOL, atol=TOL * np.abs(ref[:2]).max())


def test_noalloc_clamped_grid_then_smaller_calls_allocate_nothing():
    import torch
    rng = np.random.default_rng(7)
    # 32 x 32 x 256 cells x 2 trajectories: 524,288 cells per call, twice the 262,144 that 1024 blocks of
    # 256 threads cover in one pass, so the first stage loops over its grid stride
    big = (rng.standard_normal((2, 2, 262144)) + 1j * rng.standard_normal((2, 2, 262144))) * 0.5
    small = (rng.standard_normal((1, 2, 4096)) + 1j * rng.standard_normal((1, 2, 4096))) * 2.0
    mid = (rng.standard_normal((3, 2, 32768)) + 1j * rng.standard_normal((3, 2, 32768)))
    dV = 0.37
    d_big = torch.from_numpy(big.view(np.float64).reshape(-1).copy()).cuda()
    d_small = torch.from_numpy(small.view(np.float64).reshape(-1).copy()).cuda()
    d_mid = torch.from_numpy(mid.view(np.float64).reshape(-1).copy()).cuda()
    out = torch.empty(4, dtype=torch.float64, device="cuda")
    L = lib()

    def call(d, cells, ne):
        out.fill_(float("nan"))
        st = L.bec_moments_device_noalloc(C.c_void_p(d.data_ptr()), cells, ne, dV, C.c_void_p(out.data_ptr()), None)
        torch.cuda.synchronize()
        return st, out.cpu().numpy()

    assert call(d_small, 4096, 1)[0] == BEC_OK           # warm-up: loads the device code
    free0 = torch.cuda.mem_get_info()[0]
    for d, psi, cells, ne in ((d_big, big, 262144, 2), (d_small, small, 4096, 1), (d_mid, mid, 32768, 3),
                              (d_big, big, 262144, 2), (d_small, small, 4096, 1)):
        st, got = call(d, cells, ne)
        assert st == BEC_OK
        ref = _numpy_moments(psi, dV)
        np.testing.assert_allclose(got, ref, rtol=TOL, atol=TOL * np.abs(ref[:2]).max())
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_bad_sizes():
    import torch
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    L = lib()
    big = 1 << 20
    assert L.bec_moments_device_noalloc(C.c_void_p(buf.data_ptr()), big, big, 1.0, C.c_void_p(out.data_ptr()),
                                        None) == BEC_ERR_INVALID_ARG
    assert L.bec_moments_device_noalloc(None, 4, 1, 1.0, C.c_void_p(out.data_ptr()), None) == BEC_ERR_INVALID_ARG
    assert L.bec_moments_device_noalloc(C.c_void_p(buf.data_ptr()), 0, 1, 1.0, C.c_void_p(out.data_ptr()),
                                        None) == BEC_ERR_INVALID_ARG
    assert L.bec_moments_device_noalloc(C.c_void_p(buf.data_ptr()), 2, 1, 0.0, C.c_void_p(out.data_ptr()),
                                        None) == BEC_ERR_INVALID_ARG
    torch.cuda.synchronize()
