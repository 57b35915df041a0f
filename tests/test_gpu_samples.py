"""Moments-only samples of bec_run on the batched path.

Between steady steps the second half kick of the last step is still pending. It multiplies every
k-space amplitude of both components by the same unit-modulus factor. So the populations and
conj(a) b summed over a trajectory can be read off the stored state without ending the step. These
samples must agree with the moments of a pass that does end the step: bec_run with axial profiles
requested, and bec_moments_now (Engine.moments) after bec_evolve. They agree to FP32 rounding, because ending the
step splits the kick into two FP32 multiplications.
"""
import numpy as np
import pytest

from bec_b200.configs import rb87_params
from bec_b200.engine import BEC_PATH_FP32_BATCHED, Engine

pytestmark = pytest.mark.gpu


def thomas_fermi(d):
    x = -d.xmax + d.dx * np.arange(d.nvx)
    y = (-d.ymax + d.dy * np.arange(d.nvy)) if d.nvy > 1 else np.zeros(1)
    z = -d.zmax + d.dz * np.arange(d.nvz)
    V = (x[None, None, :] ** 2 + y[None, :, None] ** 2 + z[:, None, None] ** 2 / d.lambda_ ** 2) / 2
    return np.sqrt(np.maximum(d.mu - V, 0.0) / d.g11).reshape(-1).astype(np.complex128)


def groups():
    out = []
    for i, (grid, ne) in enumerate([((8, 8, 64), 3), ((16, 16, 128), 2), ((32, 32, 256), 1), ((32, 1, 128), 2)]):
        out.append(rb87_params(N=15000.0 + 9000.0 * i, grid=grid, ne=ne, noise=True, seed=31 + i))
    return out


def started():
    eng = Engine(groups(), path=BEC_PATH_FP32_BATCHED)
    eng.init_groups(range(eng.n_groups), [thomas_fermi(d) for d in eng.derived])
    eng.start_evolution()
    return eng


def assert_moments_close(a, b):
    """a, b: [..., 5] rows (t, na, nb, s_re, s_im)."""
    np.testing.assert_array_equal(a[..., 0], b[..., 0])
    na, nb = b[..., 1], b[..., 2]
    np.testing.assert_allclose(a[..., 1], na, rtol=1e-5)
    np.testing.assert_allclose(a[..., 2], nb, rtol=1e-5)
    scale = np.sqrt(na * nb)
    assert np.max(np.abs(a[..., 3] - b[..., 3]) / scale) < 1e-5
    assert np.max(np.abs(a[..., 4] - b[..., 4]) / scale) < 1e-5


def test_stored_state_samples_match_step_ending_samples():
    eng = started()
    fast = eng.run(24, sample_every=6)           # moments only: samples of the stored state
    eng.close()
    eng = started()
    slow, _ = eng.run(24, sample_every=6, axial=True)   # axial requested: observing passes end the steps
    eng.close()
    assert fast.shape == slow.shape == (4, 4, 5)
    assert_moments_close(fast, slow)


def test_stored_state_samples_match_moments_now():
    eng = started()
    fast = eng.run(10, sample_every=5, pi_pulse_step=5)
    eng.close()
    eng = started()
    ref = []
    for k in range(2):
        eng.evolve(5)
        ref.append(eng.moments())
        if k == 0:
            eng.pulse(np.pi)
    eng.close()
    assert_moments_close(fast, np.array(ref))
