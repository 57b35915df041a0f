"""The warm start's learned basis and its stopping rule.

CPU: the proper orthogonal decomposition and projection helpers on a synthetic two-parameter
family. GPU: the BEC_GS_MU_RESIDUAL rule of both device paths against the oracle, the device
projection on an installed basis against the host projection of the same profiles, warm starts
synthesised from that basis, and the whole pipeline (POD basis + MLP) on a small grid."""
import numpy as np
import pytest

from bec_b200 import warmstart as W
from bec_b200._abi import BEC_GS_FIXED_STEPS, BEC_GS_MU_RESIDUAL
from bec_b200.configs import rb87_params
from parity_util import record


def _family(n, seed, m=2000):
    rng = np.random.default_rng(seed)
    x = np.linspace(-1, 1, m)
    a = rng.uniform(-0.2, 0.2, n)
    w = rng.uniform(0.1, 0.2, n)
    return np.exp(-((x[None] - a[:, None]) / w[:, None]) ** 2)


def test_pod_basis_reconstructs_held_out_members():
    basis, sv = W.pod_basis(_family(300, 0), nb=40)
    nb = basis.shape[0]            # modes below the eigenvalue floor are dropped
    assert 10 < nb <= 40 and basis.shape[1] == 2000 and basis.dtype == np.float32
    assert np.all(np.diff(sv) <= 0)
    held = _family(20, 1)
    c = W.project(basis, held)
    assert c.shape == (20, 64) and np.all(c[:, nb:] == 0)
    rec = c[:, :nb] @ basis.astype(np.float64)
    assert np.linalg.norm(rec - held) / np.linalg.norm(held) < 1e-3


def test_pod_basis_drops_null_modes():
    prof = np.tile(_family(1, 2), (10, 1)) * np.linspace(1, 2, 10)[:, None]   # rank 1 around the mean
    basis, _ = W.pod_basis(prof, nb=64)
    assert basis.shape[0] == 2
    assert np.allclose(np.linalg.norm(basis.astype(np.float64), axis=1), 1.0, atol=1e-6)


def test_features_are_normalised_over_the_training_range():
    ps = W.sample_params(64, 0, grid=(8, 8, 64))
    F = W.raw_features(ps)
    assert F.shape == (64, 6)
    d = W.derive(ps[0])
    assert F[0, 0] == pytest.approx(np.log(d.mu)) and F[0, 1] == pytest.approx(np.log(d.lambda_))
    ws = W.WarmStart(None, F.min(axis=0), F.max(axis=0), 0.0, 1.0)
    f = ws.features(ps)
    assert np.all(np.abs(f) <= 1.0 + 1e-6) and np.allclose(f.min(axis=0), -1) and np.allclose(f.max(axis=0), 1)


# ---------------------------------------------------------------------------- GPU
def _oracle():
    from oracle import oracle as O
    return O


@pytest.mark.gpu
def test_plain_fp64_mu_residual_rule_matches_oracle():
    from bec_b200.engine import BEC_PATH_FP64_PLAIN, Engine
    O = _oracle()
    p = rb87_params(N=30000, grid=(8, 8, 64))
    eng = Engine([p], path=BEC_PATH_FP64_PLAIN)
    psi, rep = eng.ground_state(0, mode=BEC_GS_MU_RESIDUAL, max_steps=20000, tol=1e-6, check_every=20)
    psi_o, rep_o = O.ground_state(p, mode=BEC_GS_MU_RESIDUAL, max_steps=20000, tol=1e-6, check_every=20)
    assert rep.converged and rep.steps == rep_o.steps
    assert rep.step_residual == pytest.approx(rep_o.step_residual, rel=1e-8)
    assert rep.mu == pytest.approx(rep_o.mu, rel=1e-10)


@pytest.mark.gpu
def test_batched_mu_residual_rule_matches_oracle():
    from bec_b200.engine import BEC_PATH_FP32_BATCHED, Engine
    O = _oracle()
    ps = [rb87_params(N=30000, grid=(16, 16, 128)), rb87_params(N=90000, grid=(16, 16, 128), fz=12.0)]
    eng = Engine(ps, path=BEC_PATH_FP32_BATCHED)
    _, _, reps = eng.ground_state_coeffs(mode=BEC_GS_MU_RESIDUAL, max_steps=20000, tol=1e-6, check_every=20,
                                         want_coef=False)
    for p, r in zip(ps, reps):
        _, ro = O.ground_state(p, mode=BEC_GS_MU_RESIDUAL, max_steps=20000, tol=1e-6, check_every=20)
        assert r.converged and abs(r.steps - ro.steps) <= 20
        assert r.step_residual < 1e-5
        _, rf = O.ground_state(p, mode=BEC_GS_FIXED_STEPS, max_steps=r.steps)
        assert r.mu == pytest.approx(rf.mu, rel=5e-6)     # FP32 fixed point vs FP64 after 1000+ steps


@pytest.mark.gpu
def test_installed_basis_projection_and_warm_start():
    from bec_b200.engine import BEC_PATH_FP32_BATCHED, Engine
    grid = (16, 16, 128)
    ps = W.sample_params(24, 11, grid=grid)
    kw = dict(mode=BEC_GS_MU_RESIDUAL, max_steps=20000, tol=1e-6, check_every=20)
    eng = Engine(ps, path=BEC_PATH_FP32_BATCHED)
    _, prof, cold = eng.ground_state_coeffs(want_coef=False, want_profiles=True, **kw)
    basis, _ = W.pod_basis(prof[:16], nb=16)
    eng.set_warmstart_basis(grid, basis)
    # device projection of the same kind of states against the host projection of their profiles
    coef, prof2, _ = eng.ground_state_coeffs(want_profiles=True, **kw)
    host = W.project(basis, prof2)
    assert np.all(coef[:, basis.shape[0]:] == 0)
    assert np.linalg.norm(coef - host) / np.linalg.norm(host) < 1e-4
    # held-out sets warm-started from their own projections stop within a few checks
    held = list(range(16, 24))
    eng2 = Engine([ps[i] for i in held], path=BEC_PATH_FP32_BATCHED)
    eng2.set_warmstart_basis(grid, basis)
    _, _, warm = eng2.ground_state_coeffs(coef_in=host[held], want_coef=False, **kw)
    cold_steps = np.mean([cold[i].steps for i in held])
    warm_steps = np.mean([r.steps for r in warm])
    assert all(r.converged for r in warm)
    assert warm_steps <= 80 and cold_steps >= 5 * warm_steps
    for i, r in zip(held, warm):
        assert r.mu == pytest.approx(cold[i].mu, rel=2e-5)
    # removing the table restores the analytic basis
    eng.set_warmstart_basis(grid, None)


@pytest.mark.gpu
def test_warm_start_pipeline_beats_cold_start():
    out = W.run(n_train=512, n_eval=32, n_pod=128, seed=5, train_steps=1500, tol=1e-6, grid=(16, 16, 128),
                log=lambda *a: None)
    record("warm_start_pipeline_16x16x128", speedup_steps=out["speedup_steps"],
           mu_rel_diff_max=out["mu_rel_diff_max"])
    assert out["cold_converged"] == 1.0 and out["warm_converged"] == 1.0
    assert out["speedup_steps"] > 3.0
    assert out["mu_rel_diff_max"] < 2e-5
