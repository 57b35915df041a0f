"""Finite-duration Rabi pulses (bec_pulse_finite) against the oracle's composition
of the same Strang splitting, and the resonant Rabi transfer they must produce."""
import numpy as np
import pytest

from bec_b200 import observables as OBS
from bec_b200.configs import copy_params, rb87_params
from bec_b200.engine import BEC_PATH_FP32_BATCHED, BEC_PATH_FP64_PLAIN, Engine
from oracle import oracle as O
from parity_util import moments_rel_err, rel_state_err

pytestmark = pytest.mark.gpu


def _oracle_finite(e, rabi_hz, duration, phi, dt):
    n = max(1, int(np.floor(duration / dt + 0.5)))     # llround: halves round away from zero
    half = 0.5 * 2 * np.pi * rabi_hz * duration / n
    for _ in range(n):
        e.pulse(half, phi)
        e.evolve(1)
        e.pulse(half, phi)


@pytest.mark.parametrize("path", [BEC_PATH_FP64_PLAIN, BEC_PATH_FP32_BATCHED])
def test_finite_pulse_matches_oracle(path):
    p = rb87_params(N=20000, grid=(8, 8, 64), ne=2, noise=True, seed=4, detuning=-41.0)
    gs, _ = O.ground_state(copy_params(p, ne=1), max_steps=100)
    eng = Engine([p], path=path)
    eng.init_group(0, gs)
    e = O.OracleEnsemble(p)
    e.init(gs)
    eng.pulse_finite(500.0, 0.5e-3, 0.3)      # 12.5 steps of 40 us -> 13 substeps
    _oracle_finite(e, 500.0, 0.5e-3, 0.3, p.dt_evo)
    eng.evolve(10)
    e.evolve(10)
    tol = 1e-10 if path == BEC_PATH_FP64_PLAIN else 1e-4
    assert max(moments_rel_err(eng.moments()[0], e.moments())) < tol
    for t in range(p.ne):
        assert rel_state_err(eng.get_state(0, t), e.get_state(t)) < (1e-10 if path == BEC_PATH_FP64_PLAIN else 2e-4)


def test_resonant_pi_pulse_transfers_population():
    """A short resonant pi pulse (Omega = 2 pi x 5 kHz >> mu / h) moves nearly all atoms to |2>."""
    p = rb87_params(N=5000, grid=(16, 16, 128), ne=1, noise=False, losses=False, dt_evo=1e-6)
    eng = Engine([p], path=BEC_PATH_FP32_BATCHED)
    gs, _ = eng.ground_state(0, max_steps=400)
    eng.init_group(0, gs)
    d = eng.derived[0]
    eng.pulse_finite(5000.0, 1.0e-4, 0.0)    # Omega t = pi
    m = eng.moments()[0]
    n1, n2 = OBS.populations(m, d, 1)
    assert n2 / (n1 + n2) > 0.99
