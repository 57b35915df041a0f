"""Largest configuration, empty runs and misuse, through the C ABI.

At the full size of the spin-echo configuration (1024 trajectories of 32 x 32 x 256, 4.3 GB of
state) no oracle run is affordable, so the check is a size-independent property: without losses
every pass is unitary (the kinetic and nonlinear factors have unit modulus), so the total population
of every trajectory stays at its initial value to FP32 rounding.
"""
import numpy as np
import pytest

from bec_b200.configs import rb87_params
from bec_b200.engine import BEC_PATH_FP32_BATCHED, BecError, Engine

pytestmark = pytest.mark.gpu


def thomas_fermi(d):
    x = -d.xmax + d.dx * np.arange(d.nvx)
    y = (-d.ymax + d.dy * np.arange(d.nvy)) if d.nvy > 1 else np.zeros(1)
    z = -d.zmax + d.dz * np.arange(d.nvz)
    V = (x[None, None, :] ** 2 + y[None, :, None] ** 2 + z[:, None, None] ** 2 / d.lambda_ ** 2) / 2
    return np.sqrt(np.maximum(d.mu - V, 0.0) / d.g11).reshape(-1).astype(np.complex128)


def test_full_size_spin_echo_conserves_population():
    p = rb87_params(N=70000.0, grid=(32, 32, 256), ne=1024, noise=True, losses=False, seed=4)
    eng = Engine([p], path=BEC_PATH_FP32_BATCHED)
    assert eng.n_traj == 1024
    eng.init_groups([0], [thomas_fermi(eng.derived[0]).astype(np.complex64)])
    eng.start_evolution()
    mom = eng.run(24, sample_every=8, pi_pulse_step=12)
    traj = eng.traj_moments()
    eng.close()
    assert mom.shape == (3, 1, 5) and np.all(np.isfinite(mom))
    total = mom[:, 0, 1] + mom[:, 0, 2]
    np.testing.assert_allclose(total, total[0], rtol=1e-5)
    # every trajectory on its own, and the ensemble sum is theirs
    assert traj.shape == (1024, 5) and np.all(np.isfinite(traj))
    np.testing.assert_allclose(traj[:, 1].sum() + traj[:, 2].sum(), total[-1], rtol=1e-5)
    # after the opening pi/2 pulse both components hold atoms in every trajectory
    assert np.all(traj[:, 1] > 0) and np.all(traj[:, 2] > 0)


def small_engine():
    groups = [rb87_params(N=20000.0, grid=(8, 8, 64), ne=2, noise=True, seed=5),
              rb87_params(N=30000.0, grid=(16, 16, 128), ne=1, noise=True, seed=6)]
    eng = Engine(groups, path=BEC_PATH_FP32_BATCHED)
    return eng, groups


def test_zero_steps_change_nothing():
    eng, groups = small_engine()
    eng.init_groups(range(len(groups)), [thomas_fermi(d) for d in eng.derived])
    eng.start_evolution()
    eng.evolve(3)
    before = [eng.get_state(g, t) for g, p in enumerate(groups) for t in range(p.ne)]
    step = eng.step_index
    eng.evolve(0)
    mom = eng.run(0)
    assert mom.shape == (0, len(groups), 5)
    assert eng.step_index == step
    after = [eng.get_state(g, t) for g, p in enumerate(groups) for t in range(p.ne)]
    for a, b in zip(before, after):
        np.testing.assert_array_equal(a, b)
    eng.close()


def test_misuse_is_reported():
    eng, groups = small_engine()
    with pytest.raises(BecError):
        eng.start_evolution()                 # no group initialised yet
    with pytest.raises(BecError):
        eng.evolve(1)
    eng.init_group(0, thomas_fermi(eng.derived[0]))
    with pytest.raises(BecError):
        eng.evolve(1)                         # group 1 still missing
    eng.close()
    for grid in [(12, 12, 64), (8, 8, 1024), (64, 64, 64)]:
        # not a power of two; pencils longer than the batched z pass holds; planes larger than it holds
        with pytest.raises(BecError):
            Engine([rb87_params(N=20000.0, grid=grid, ne=1)], path=BEC_PATH_FP32_BATCHED)
