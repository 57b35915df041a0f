"""Checkpoint and resume, and failure detection driven from the host.

* A raw checkpoint (bec_checkpoint_save / bec_checkpoint_load) restored into a fresh context resumes
  the run bit for bit: the loss noise continues the same Philox stream because the step counter
  travels with the state, and a pending half kick or pulse stays pending.
* Resuming from x-space states (bec_get_state -> bec_set_state) plus bec_set_step_index matches the
  uninterrupted run to FP32 rounding; without the step index the noise stream restarts and the runs
  part by far more.
* Failures are made on the host, never on the GPU: a NaN planted through bec_set_state makes the next
  sample return BEC_ERR_NUMERICAL; a device byte limit (BEC_DEVICE_BYTES_LIMIT) makes context creation
  fail with BEC_ERR_OUT_OF_MEMORY before any allocation reaches the device, and the next context works.
"""
import numpy as np
import pytest

from bec_b200._abi import BEC_ERR_INVALID_ARG, BEC_ERR_NUMERICAL, BEC_ERR_OUT_OF_MEMORY
from bec_b200.configs import copy_params, rb87_params
from bec_b200.engine import BEC_PATH_FP32_BATCHED, BEC_PATH_FP64_PLAIN, BecError, Engine
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PATHS = [BEC_PATH_FP64_PLAIN, BEC_PATH_FP32_BATCHED]


def _groups():
    return [rb87_params(N=20000, grid=(8, 8, 64), ne=2, noise=True, seed=41),
            rb87_params(N=35000, grid=(16, 16, 128), ne=1, noise=True, seed=42)]


def _started(groups, path):
    eng = Engine(groups, path=path)
    for g, p in enumerate(groups):
        gs, _ = O.ground_state(copy_params(p, ne=1), max_steps=60)
        eng.init_group(g, gs)
    eng.start_evolution()
    return eng


def _states(eng, groups):
    return [eng.get_state(g, t) for g, p in enumerate(groups) for t in range(p.ne)]


@pytest.mark.parametrize("path", PATHS)
def test_raw_checkpoint_resumes_bit_identically(path):
    groups = _groups()
    ref = _started(groups, path)
    ref.evolve(30)
    ref.pulse(np.pi, 0.3)                       # pending at the checkpoint on the batched path
    blob = ref.checkpoint()
    m_ref = ref.run(40, sample_every=20, pi_pulse_step=25)
    s_ref = _states(ref, groups)

    res = Engine(groups, path=path)
    res.restore(blob)
    assert res.step_index == ref.step_index - 40 and res.evolution_steps == 30
    m_res = res.run(40, sample_every=20, pi_pulse_step=25)
    np.testing.assert_array_equal(m_res, m_ref)
    for a, b in zip(_states(res, groups), s_ref):
        np.testing.assert_array_equal(a, b)
    assert res.step_index == ref.step_index


def test_checkpoint_of_another_layout_is_rejected():
    groups = _groups()
    eng = _started(groups, BEC_PATH_FP32_BATCHED)
    blob = eng.checkpoint()
    other = Engine([copy_params(groups[0], seed=7), groups[1]], path=BEC_PATH_FP32_BATCHED)
    with pytest.raises(BecError) as ei:
        other.restore(blob)
    assert ei.value.status == BEC_ERR_INVALID_ARG
    plain = Engine(groups, path=BEC_PATH_FP64_PLAIN)
    with pytest.raises(BecError):
        plain.restore(blob)
    with pytest.raises(BecError):
        Engine(groups, path=BEC_PATH_FP32_BATCHED).restore(blob[:100])


def test_xspace_resume_with_step_index():
    groups = _groups()
    ref = _started(groups, BEC_PATH_FP32_BATCHED)
    ref.evolve(25)
    saved = _states(ref, groups)
    step, evo = ref.step_index, ref.evolution_steps
    m_ref = ref.run(30, sample_every=30)[-1]
    s_ref = _states(ref, groups)

    def resumed(set_index):
        eng = Engine(groups, path=BEC_PATH_FP32_BATCHED)
        k = 0
        for g, p in enumerate(groups):
            for t in range(p.ne):
                eng.set_state(g, t, saved[k])
                k += 1
        if set_index:
            eng.set_step_index(step, evo)
        m = eng.run(30, sample_every=30)[-1]
        return m, _states(eng, groups)

    m_ok, s_ok = resumed(True)
    m_bad, s_bad = resumed(False)
    np.testing.assert_allclose(m_ok[:, 0], m_ref[:, 0], rtol=1e-12)
    err_ok = max(np.abs(a - b).max() / np.abs(b).max() for a, b in zip(s_ok, s_ref))
    err_bad = max(np.abs(a - b).max() / np.abs(b).max() for a, b in zip(s_bad, s_ref))
    assert err_ok < 2e-5
    assert err_bad > 20 * err_ok


@pytest.mark.parametrize("path", PATHS)
def test_planted_nan_is_reported_as_numerical_error(path):
    groups = _groups()
    eng = _started(groups, path)
    eng.evolve(5)
    ab = eng.get_state(1, 0)
    ab[0, 1234] = np.nan
    eng.set_state(1, 0, ab)
    with pytest.raises(BecError) as ei:
        eng.run(10, sample_every=5)
    assert ei.value.status == BEC_ERR_NUMERICAL
    # the other context on the device is unaffected
    ok = _started(groups, path)
    assert np.isfinite(ok.run(5, sample_every=5)).all()


def test_device_byte_limit_fails_creation_then_recovers(monkeypatch):
    groups = _groups()
    monkeypatch.setenv("BEC_DEVICE_BYTES_LIMIT", str(1 << 20))
    for path in PATHS:
        with pytest.raises(BecError) as ei:
            Engine(groups, path=path)
        assert ei.value.status == BEC_ERR_OUT_OF_MEMORY
    monkeypatch.setenv("BEC_DEVICE_BYTES_LIMIT", str(1 << 34))
    eng = _started(groups, BEC_PATH_FP32_BATCHED)
    assert np.isfinite(eng.run(5, sample_every=5)).all()
    monkeypatch.delenv("BEC_DEVICE_BYTES_LIMIT")
    eng2 = _started(groups, BEC_PATH_FP32_BATCHED)
    np.testing.assert_array_equal(eng2.run(5, sample_every=5), _started(groups, BEC_PATH_FP32_BATCHED).run(5, sample_every=5))
