"""The reference's stored GPU curve (data/gpu_sp_30k.yaml) as a shape check,
and the FP64 oracle's curve of the same run as an end-to-end fixture.

The stored curve's loss and detuning parameters were never recorded, so it
pins the physics loosely: with the workload's Rb-87 loss rates the oracle
follows it within 0.006 to 0.1 s and 0.035 to 0.3 s (first dip and revival).
The oracle's own curve (generated by tests/golden/make_golden.py) checks the
batched FP32 engine over all 15000 steps against an FP64-parity bound of
1e-3 in visibility."""
import json
import os

import numpy as np
import pytest

from bec_b200 import observables as OBS
from bec_b200._abi import BEC_GS_REFERENCE_E
from bec_b200.configs import rb87_params
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "gpu_sp_30k.json")))


def _params():
    return rb87_params(N=30000, grid=(16, 16, 128), ne=1, noise=False)


def test_fixture_consistency():
    ref, orc = GOLD["reference"], GOLD["oracle"]
    assert len(ref["t"]) == len(orc["t"]) == 61
    np.testing.assert_allclose(orc["t"], ref["t"], atol=1e-9)
    assert ref["visibility"][0] == 1.0 and abs(orc["visibility"][0] - 1.0) < 1e-12


def test_oracle_curve_shape_matches_reference_curve():
    """Window agreement and the timing of the first dip and revival."""
    t = np.array(GOLD["reference"]["t"])
    ref = np.array(GOLD["reference"]["visibility"])
    orc = np.array(GOLD["oracle"]["visibility"])
    assert np.abs(orc - ref)[t <= 0.1 + 1e-9].max() < 0.01
    assert np.abs(orc - ref)[t <= 0.3 + 1e-9].max() < 0.035
    dip = slice(5, 26)          # 0.05 .. 0.25 s
    rev = slice(25, 40)         # 0.25 .. 0.39 s
    assert abs(t[dip][np.argmin(ref[dip])] - t[dip][np.argmin(orc[dip])]) <= 0.02 + 1e-9
    assert abs(t[rev][np.argmax(ref[rev])] - t[rev][np.argmax(orc[rev])]) <= 0.03 + 1e-9
    assert abs(ref[dip].min() - orc[dip].min()) < 0.03


def test_oracle_regenerates_first_samples():
    """The committed oracle curve is what the oracle computes now (first 1250 steps)."""
    p = _params()
    gs, rep = O.ground_state(p, mode=BEC_GS_REFERENCE_E, max_steps=20000)
    assert rep.steps == GOLD["oracle"]["ground_state_steps"]
    e = O.OracleEnsemble(p)
    e.init(gs)
    e.start_evolution()
    for k in range(1, 6):
        e.evolve(250, 0)
        m = e.moments()
        np.testing.assert_allclose(m, GOLD["oracle"]["moments"][k], rtol=1e-10)


@pytest.mark.gpu
def test_engine_fp32_full_curve_against_oracle():
    """15000 FP32 steps of the batched engine: visibility within 1e-3 of the FP64 oracle
    and the reference curve's shape."""
    from bec_b200.engine import BEC_PATH_FP32_BATCHED, Engine
    p = _params()
    eng = Engine([p], path=BEC_PATH_FP32_BATCHED)
    gs, rep = eng.ground_state(0, mode=BEC_GS_REFERENCE_E, max_steps=20000)
    assert rep.steps == GOLD["oracle"]["ground_state_steps"]
    eng.init_group(0, gs)
    eng.start_evolution()
    mom = eng.run(15000, sample_every=250)[:, 0]
    d = eng.derived[0]
    vis = np.array([OBS.visibility(m, d, 1) for m in mom])
    orc = np.array(GOLD["oracle"]["visibility"][1:])
    err = np.abs(vis - orc).max()
    from parity_util import record
    record("golden_fp32_15000", vis_err=err)
    assert err < 1e-3
    ref = np.array(GOLD["reference"]["visibility"][1:])
    t = np.array(GOLD["reference"]["t"][1:])
    assert np.abs(vis - ref)[t <= 0.3 + 1e-9].max() < 0.035
