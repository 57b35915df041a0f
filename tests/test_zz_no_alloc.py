"""bec_moments_device_noalloc: moments of states in the caller's device memory,
computed without any device allocation (for callers that cannot let the
library call cudaMalloc: hosts that own all device memory through their own
pool, and loops that must never block on an allocation).

Checked through the C ABI against bec_moments_now of a context holding the
same states, on two calls in a row with different inputs and sizes (the
second call runs over the scratch contents the first one left behind).
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


def test_noalloc_moments_match_context_moments_twice():
    cases = [((16, 16, 128), 3, 1), ((8, 8, 64), 2, 2)]
    for grid, ne, seed in cases:
        psi, cells, dV, expect = _states(grid, ne, seed)
        st, got = _noalloc(psi, cells, ne, dV)
        assert st == BEC_OK
        np.testing.assert_allclose(got, expect[1:], rtol=TOL, atol=TOL * np.abs(expect[1:3]).max())


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
