"""Batched FP32 imaginary-time ground states (bec_ground_state_batch on the
batched path) against the CPU FP64 oracle's calculateSteadyState restatement.

Tolerance: FP32 states within 2e-5 of the oracle's max |psi| after a fixed
step count (imaginary time damps rounding instead of amplifying it); mu from
the FP64 measures within 1e-6 relative after 400 steps and 5e-6 after 1000+
(the FP32 loop's own fixed point); the mu stopping rule fires within one check
interval of the oracle's."""
import ctypes as C

import numpy as np
import pytest

from bec_b200._abi import BEC_GS_FIXED_STEPS, BEC_GS_MU, BEC_GS_MU_RESIDUAL, BecGsOpts, BecGsReport
from bec_b200.configs import rb87_params
from bec_b200.engine import BEC_PATH_FP32_BATCHED, Engine, lib
from oracle import oracle as O
from parity_util import record, rel_state_err

pytestmark = pytest.mark.gpu

GROUPS = [
    rb87_params(N=15000, grid=(8, 8, 64), fx=90.0, fy=90.0),
    rb87_params(N=40000, grid=(16, 16, 128), fz=12.8),
    rb87_params(N=30000, grid=(16, 16, 128)),
    rb87_params(N=70000, grid=(32, 32, 256), fx=101.0, fy=101.0, fz=11.0),
]


def batch_gs(eng, groups, mode, max_steps, tol=1e-6, check_every=10, warm=None):
    n = len(groups)
    o = BecGsOpts()
    o.mode, o.max_steps, o.check_every, o.tol = mode, max_steps, check_every, tol
    ws = None
    if warm is not None:
        ws = np.ascontiguousarray(warm, dtype=np.complex128)
        o.warm_start = ws.ctypes.data_as(C.POINTER(C.c_double))
    outs = [np.zeros(eng.derived[g].cells, dtype=np.complex128) for g in groups]
    ptrs = (C.POINTER(C.c_double) * n)(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in outs])
    idx = (C.c_int32 * n)(*groups)
    reps = (BecGsReport * n)()
    st = lib().bec_ground_state_batch(eng._h, n, idx, C.byref(o), ptrs, reps)
    eng._check(st, "bec_ground_state_batch")
    return outs, list(reps)


def test_batched_fixed_steps_match_oracle():
    eng = Engine(GROUPS, path=BEC_PATH_FP32_BATCHED)
    outs, reps = batch_gs(eng, list(range(len(GROUPS))), BEC_GS_FIXED_STEPS, 400)
    worst = 0.0
    for g, p in enumerate(GROUPS):
        psi_o, rep_o = O.ground_state(p, mode=BEC_GS_FIXED_STEPS, max_steps=400)
        err = rel_state_err(outs[g], psi_o)
        worst = max(worst, err)
        assert reps[g].steps == 400
        assert reps[g].N == pytest.approx(p.N, rel=1e-5)
        assert reps[g].mu == pytest.approx(rep_o.mu, rel=1e-6)
    record("gs_batched_fixed400", state_err=worst)
    assert worst < 2e-5


def test_batched_every_supported_shape_matches_oracle():
    """Every grid the batched loop takes (square 8, 16 and 32 planes by nz = 64, 128 and 256), nine classes in
    one context: 100 fixed steps against the oracle."""
    groups = [rb87_params(N=20000 + 5000 * k, grid=(n, n, nz), fz=11.0 + k)
              for k, (n, nz) in enumerate((n, nz) for n in (8, 16, 32) for nz in (64, 128, 256))]
    eng = Engine(groups, path=BEC_PATH_FP32_BATCHED)
    outs, reps = batch_gs(eng, list(range(len(groups))), BEC_GS_FIXED_STEPS, 100)
    worst = 0.0
    for g, p in enumerate(groups):
        psi_o, rep_o = O.ground_state(p, mode=BEC_GS_FIXED_STEPS, max_steps=100)
        err = rel_state_err(outs[g], psi_o)
        worst = max(worst, err)
        assert reps[g].steps == 100
        assert reps[g].mu == pytest.approx(rep_o.mu, rel=1e-6), (p.nvx, p.nvz)
        assert err < 2e-5, (p.nvx, p.nvz, err)
    record("gs_batched_every_shape_fixed100", state_err=worst)


def test_batched_mu_rule_matches_oracle():
    sel = [0, 2]
    eng = Engine(GROUPS, path=BEC_PATH_FP32_BATCHED)
    outs, reps = batch_gs(eng, sel, BEC_GS_MU, 6000, tol=1e-6, check_every=20)
    for k, g in enumerate(sel):
        psi_o, rep_o = O.ground_state(GROUPS[g], mode=BEC_GS_MU, max_steps=6000, tol=1e-6, check_every=20)
        assert reps[k].converged == 1 and rep_o.converged == 1
        assert abs(reps[k].steps - rep_o.steps) <= 20
        # the state and mu still move by up to ~tol per check when the rule stops, so compare with the
        # oracle at the same step count; after 1000+ steps the FP32 loop's fixed point sits a few 1e-6
        # from the FP64 one
        psi_f, rep_f = O.ground_state(GROUPS[g], mode=BEC_GS_FIXED_STEPS, max_steps=reps[k].steps)
        assert rel_state_err(outs[k], psi_f) < 1e-4
        assert reps[k].mu == pytest.approx(rep_f.mu, rel=5e-6)


def test_batched_warm_start_needs_fewer_steps():
    # the mu-only rule can stop a cold start at mu's minimum, before the state is stationary, so the
    # comparison uses the rule that also bounds the fixed-point residual
    p = [GROUPS[2]]
    eng = Engine(p, path=BEC_PATH_FP32_BATCHED)
    psi, rep = batch_gs(eng, [0], BEC_GS_MU_RESIDUAL, 6000, tol=1e-6, check_every=20)
    _, rep2 = batch_gs(eng, [0], BEC_GS_MU_RESIDUAL, 6000, tol=1e-6, check_every=20, warm=psi[0])
    assert rep[0].converged and rep2[0].converged
    assert rep2[0].steps <= 60 and rep[0].steps > 400
