"""Parity of the CUDA engine (called through the C ABI) against the CPU FP64 oracle.

Tolerances:
  FP64 plain path ........ 1e-10 relative (states and moments), the bar of the
                           reference's own CPU path restated in FP64.
  FP32 batched path ...... per-trajectory states within FP32_STATE_* of the
                           oracle's max |psi|; moments within FP32_MOM relative;
                           visibility within 1e-4 absolute. Over the 2500 steps
                           of the 2D configuration the dynamics amplify rounding
                           (the FP64 path drifts from 1e-16 to ~6e-13 there), so
                           the FP32 state bound is 3e-2 and the moment bound 1e-3
                           for that run; ensemble visibility stays within 1e-4.
"""
import numpy as np
import pytest

from bec_b200 import observables as OBS
from bec_b200._abi import BEC_GS_FIXED_STEPS, BEC_GS_MU, BEC_GS_REFERENCE_E
from bec_b200.configs import slice_2d_32x128, ensemble_16x16x128, copy_params, rb87_params
from bec_b200.engine import BEC_PATH_FP32_BATCHED, BEC_PATH_FP64_PLAIN, Engine
from oracle import oracle as O
from parity_util import engine_sequence, moments_rel_err, oracle_sequence, record, rel_state_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_STATE_SHORT = 2e-4     # <= 200 steps
FP32_STATE_LONG = 3e-2      # 2500 steps
FP32_MOM = 1e-4
FP32_MOM_LONG = 1e-3        # 2500 steps
FP32_VIS = 1e-4

PATHS = [BEC_PATH_FP64_PLAIN, BEC_PATH_FP32_BATCHED]


@pytest.fixture(scope="module")
def slice_gs():
    p = slice_2d_32x128()
    psi, rep = O.ground_state(p, mode=BEC_GS_FIXED_STEPS, max_steps=2000)
    return p, psi


# ------------------------------------------------------------------ ground state
def test_fp64_ground_state_2d_slice_2000_steps(slice_gs):
    """The 2D 32x128 slice: 2000 imaginary-time steps from Thomas-Fermi."""
    p, psi_o = slice_gs
    eng = Engine([p], path=BEC_PATH_FP64_PLAIN)
    psi, rep = eng.ground_state(0, mode=BEC_GS_FIXED_STEPS, max_steps=2000)
    err = rel_state_err(psi, psi_o)
    record("gs_slice2d_fp64", state_err=err)
    assert rep.steps == 2000
    assert err < FP64_TOL
    mu_o, e_o, r_o, n_o = O.gs_measures(p, psi_o)
    assert rep.mu == pytest.approx(mu_o, rel=1e-10)
    assert rep.energy == pytest.approx(e_o, rel=1e-10)
    assert rep.N == pytest.approx(n_o, rel=1e-12)
    assert rep.residual == pytest.approx(r_o, rel=1e-6)


@pytest.mark.parametrize("path", PATHS)
def test_ground_state_modes_3d(path):
    p = rb87_params(N=30000, grid=(16, 16, 128))
    eng = Engine([p], path=path)
    psi, rep = eng.ground_state(0, mode=BEC_GS_MU, max_steps=3000, tol=1e-7, check_every=10)
    psi_o, rep_o = O.ground_state(p, mode=BEC_GS_MU, max_steps=3000, tol=1e-7, check_every=10)
    assert rep.converged and rep.steps == rep_o.steps
    assert rel_state_err(psi, psi_o) < 1e-9
    assert rep.mu == pytest.approx(rep_o.mu, rel=1e-10)
    psi2, rep2 = eng.ground_state(0, mode=BEC_GS_REFERENCE_E, max_steps=20000)
    psi2_o, rep2_o = O.ground_state(p, mode=BEC_GS_REFERENCE_E, max_steps=20000)
    assert rep2.steps == rep2_o.steps
    assert rel_state_err(psi2, psi2_o) < 1e-9


def test_ground_state_warm_start():
    p = rb87_params(N=30000, grid=(8, 8, 64))
    eng = Engine([p], path=BEC_PATH_FP32_BATCHED)
    psi, _ = eng.ground_state(0, max_steps=300)
    psi_o, _ = O.ground_state(p, max_steps=300)
    assert rel_state_err(psi, psi_o) < 1e-10
    _, cold = eng.ground_state(0, mode=BEC_GS_MU, max_steps=5000, tol=1e-6, check_every=5)
    _, warm = eng.ground_state(0, mode=BEC_GS_MU, max_steps=5000, tol=1e-6, check_every=5, warm_start=psi)
    assert cold.converged and warm.converged
    assert warm.steps < cold.steps


# ------------------------------------------------------------------ 2D 32x128 evolution
@pytest.mark.parametrize("path", PATHS)
def test_2d_slice_evolution(slice_gs, path):
    """The 2D 32x128 slice: pi/2 then 100 ms (2500 steps), no noise, samples every 250 steps."""
    p, gs = slice_gs
    mo, eo = oracle_sequence(p, gs, 2500, 250)
    me, ee = engine_sequence(p, gs, 2500, 250, path)
    assert me.shape == mo.shape
    np.testing.assert_allclose(me[:, 0], mo[:, 0], rtol=1e-12)
    tol_m = FP64_TOL if path == BEC_PATH_FP64_PLAIN else FP32_MOM_LONG
    worst_m = max(max(moments_rel_err(a, b)) for a, b in zip(me, mo))
    d = eo.d
    vis_e = [OBS.visibility(m, d, 1) for m in me]
    vis_o = [OBS.visibility(m, d, 1) for m in mo]
    vis_err = float(np.max(np.abs(np.array(vis_e) - np.array(vis_o))))
    st_err = rel_state_err(ee.get_state(0, 0), eo.get_state(0))
    record(f"slice2d_path{path}", moments_err=worst_m, vis_err=vis_err, state_err=st_err)
    assert worst_m < tol_m
    assert st_err < (FP64_TOL if path == BEC_PATH_FP64_PLAIN else FP32_STATE_LONG)
    assert vis_err < (1e-10 if path == BEC_PATH_FP64_PLAIN else FP32_VIS)


# ------------------------------------------------------------------ Wigner noise, per trajectory
@pytest.mark.parametrize("path", PATHS)
def test_wigner_noise_per_trajectory(path):
    """Philox initial noise + loss noise, 16x16x128, 3 trajectories, 150 steps: the same
    counter-based draws on both sides, so each trajectory matches."""
    p = rb87_params(N=30000, grid=(16, 16, 128), ne=3, noise=True, seed=11)
    gs, _ = O.ground_state(copy_params(p, ne=1), max_steps=300)
    mo, eo = oracle_sequence(p, gs, 150, 50)
    me, ee = engine_sequence(p, gs, 150, 50, path)
    tol_s = 1e-9 if path == BEC_PATH_FP64_PLAIN else FP32_STATE_SHORT
    worst = 0.0
    for t in range(p.ne):
        worst = max(worst, rel_state_err(ee.get_state(0, t), eo.get_state(t)))
    tm_e, tm_o = ee.traj_moments(), eo.traj_moments()
    tm_err = float(np.max(np.abs(tm_e[:, 1:3] - tm_o[:, 1:3]) / tm_o[:, 1:3]))
    record(f"noise_traj_path{path}", state_err=worst, traj_mom_err=tm_err)
    assert worst < tol_s
    assert tm_err < (1e-10 if path == BEC_PATH_FP64_PLAIN else FP32_MOM)


@pytest.mark.parametrize("path", PATHS)
def test_injected_noise_arrays(path):
    """Trajectories driven by caller-supplied initial noise arrays."""
    p = rb87_params(N=20000, grid=(8, 8, 64), ne=2, noise=True, loss_noise=False)
    d = O.derive(p)
    rng = np.random.default_rng(5)
    noise = 0.5 * (rng.standard_normal((2, 2, d.cells)) + 1j * rng.standard_normal((2, 2, d.cells)))
    gs, _ = O.ground_state(copy_params(p, ne=1), max_steps=200)
    mo, eo = oracle_sequence(p, gs, 100, 100, noise=noise)
    me, ee = engine_sequence(p, gs, 100, 100, path, noise=noise)
    tol_s = 1e-10 if path == BEC_PATH_FP64_PLAIN else FP32_STATE_SHORT
    for t in range(p.ne):
        assert rel_state_err(ee.get_state(0, t), eo.get_state(t)) < tol_s


# ------------------------------------------------------------------ uneven batch
def test_uneven_batch_fp32():
    """Mixed grids and atom numbers in one context (one launch per pass and grid class)."""
    groups = [
        rb87_params(N=15000, grid=(8, 8, 64), ne=2, noise=True, seed=1, fx=92.0, fy=92.0),
        rb87_params(N=40000, grid=(16, 16, 128), ne=1, noise=True, seed=2, fz=12.5),
        rb87_params(N=25000, grid=(32, 1, 128), ne=2, noise=True, seed=3),
        rb87_params(N=60000, grid=(8, 8, 64), ne=1, noise=False, seed=4),
    ]
    eng = Engine(groups, path=BEC_PATH_FP32_BATCHED)
    gss, ens = [], []
    for g, p in enumerate(groups):
        gs, _ = O.ground_state(copy_params(p, ne=1), max_steps=200)
        gss.append(gs)
        eng.init_group(g, gs)
        e = O.OracleEnsemble(p)
        e.init(gs)
        e.start_evolution()
        ens.append(e)
    eng.start_evolution()
    mom = eng.run(60, sample_every=30)
    for e in ens:
        e.evolve(60)
    for g, (p, e) in enumerate(zip(groups, ens)):
        mo = e.moments()
        err = moments_rel_err(mom[-1, g], mo)
        assert max(err) < FP32_MOM, (g, err)
        for t in range(p.ne):
            assert rel_state_err(eng.get_state(g, t), e.get_state(t)) < FP32_STATE_SHORT


# the register-resident shapes the other tests leave out (8, 16, 32 planes by nz = 64, 128, 256)
FAST_SHAPES = [
    rb87_params(N=15000, grid=(8, 8, 128), ne=2, noise=True, seed=31),
    rb87_params(N=20000, grid=(8, 8, 256), ne=2, noise=True, seed=32, fz=8.0),
    rb87_params(N=30000, grid=(16, 16, 256), ne=2, noise=True, seed=33),
    rb87_params(N=40000, grid=(32, 32, 64), ne=2, noise=True, seed=34, fz=30.0),
    rb87_params(N=50000, grid=(32, 32, 128), ne=2, noise=True, seed=35),
]


@pytest.fixture(scope="module")
def fast_shape_oracle():
    gss, moms, states = [], [], []
    for p in FAST_SHAPES:
        gs, _ = O.ground_state(copy_params(p, ne=1), max_steps=200)
        e = O.OracleEnsemble(p)
        e.init(gs)
        e.start_evolution()
        e.evolve(40)
        gss.append(gs)
        moms.append(e.moments())
        states.append([e.get_state(t) for t in range(p.ne)])
    return gss, moms, states


@pytest.mark.parametrize("plan", ["unfused", "unfused-tma"])
def test_register_shapes_off_the_workload(monkeypatch, fast_shape_oracle, plan):
    """The register-resident plane and pencil passes (register or TMA pencils) on the shapes the workload does
    not use, one context: states and moments against the oracle after 40 steps with noise and losses."""
    monkeypatch.setenv("BEC_STEP_PLAN", plan)
    gss, moms, states = fast_shape_oracle
    eng = Engine(FAST_SHAPES, path=BEC_PATH_FP32_BATCHED)
    for g, gs in enumerate(gss):
        eng.init_group(g, gs)
    eng.start_evolution()
    mom = eng.run(40, sample_every=20)
    worst_m, worst_s = 0.0, 0.0
    for g, p in enumerate(FAST_SHAPES):
        err = max(moments_rel_err(mom[-1, g], moms[g]))
        se = max(rel_state_err(eng.get_state(g, t), states[g][t]) for t in range(p.ne))
        worst_m, worst_s = max(worst_m, err), max(worst_s, se)
        assert err < FP32_MOM and se < FP32_STATE_SHORT, ((p.nvx, p.nvz), err, se)
    record(f"register_shapes_{plan}", moments=worst_m, state=worst_s)


UNUSUAL_GRIDS = [
    rb87_params(N=20000, grid=(16, 8, 64), ne=2, noise=True, seed=21, fy=70.0),      # nx != ny: generic plane pass
    rb87_params(N=15000, grid=(8, 8, 32), ne=2, noise=True, seed=22),                # nz = 32: generic z pass
    rb87_params(N=10000, grid=(4, 4, 512), ne=1, noise=True, seed=23, fz=6.0),       # nz = 512, 4 x 4 planes
    rb87_params(N=30000, grid=(64, 32, 16), ne=1, noise=True, seed=24, fy=60.0, fz=40.0),  # the largest plane
    rb87_params(N=25000, grid=(128, 1, 32), ne=2, noise=True, seed=25, fy=50.0),     # a wide 2D slice
]


@pytest.mark.parametrize("path", PATHS)
def test_uneven_batch_unusual_grids(path):
    """Grid shapes off the register-resident passes (nx != ny, nz of 32 and 512, a 64 x 32 plane, a 128-wide
    slice), all in one context: states and moments against the oracle after 40 steps with noise and losses."""
    groups = UNUSUAL_GRIDS
    eng = Engine(groups, path=path)
    ens = []
    for g, p in enumerate(groups):
        gs, _ = O.ground_state(copy_params(p, ne=1), max_steps=200)
        eng.init_group(g, gs)
        e = O.OracleEnsemble(p)
        e.init(gs)
        e.start_evolution()
        ens.append(e)
    eng.start_evolution()
    mom = eng.run(40, sample_every=20)
    for e in ens:
        e.evolve(40)
    worst_m, worst_s = 0.0, 0.0
    for g, (p, e) in enumerate(zip(groups, ens)):
        err = max(moments_rel_err(mom[-1, g], e.moments()))
        se = max(rel_state_err(eng.get_state(g, t), e.get_state(t)) for t in range(p.ne))
        worst_m, worst_s = max(worst_m, err), max(worst_s, se)
        if path == BEC_PATH_FP64_PLAIN:
            assert err < FP64_TOL and se < FP64_TOL, (g, err, se)
        else:
            assert err < FP32_MOM and se < FP32_STATE_SHORT, (g, err, se)
    record(f"unusual_grids_{'fp64' if path == BEC_PATH_FP64_PLAIN else 'fp32'}", moments=worst_m, state=worst_s)


# ------------------------------------------------------------------ schedule, pulses, observables
@pytest.mark.parametrize("path", PATHS)
def test_run_with_pi_pulse_and_axial(path):
    """Spin echo: pi pulse after 40 of 80 steps; samples every 20 with axial profiles."""
    p = rb87_params(N=30000, grid=(8, 8, 64), ne=2, noise=True, seed=9)
    gs, _ = O.ground_state(copy_params(p, ne=1), max_steps=200)
    mo, eo = oracle_sequence(p, gs, 80, 20, pi_pulse_step=40)
    eng = Engine([p], path=path)
    eng.init_group(0, gs)
    eng.start_evolution()
    mom, axial = eng.run(80, sample_every=20, pi_pulse_step=40, axial=True)
    tol = 1e-10 if path == BEC_PATH_FP64_PLAIN else FP32_MOM
    for a, b in zip(mom[:, 0], mo):
        assert max(moments_rel_err(a, b)) < tol
    ax_o = eo.axial()
    ax_e = axial[0][-1]
    # the last sample precedes nothing else, so it is the oracle's final state
    np.testing.assert_allclose(ax_e[:, :2], ax_o[:, :2], rtol=tol * 10, atol=tol * ax_o[:, :2].max())
    # the ratio (a - b)/(a + b) is ill-conditioned where the Wigner-subtracted density
    # a + b vanishes (the condensate's edge); compare it where a + b is resolved
    d = eo.d
    sub = p.ne * d.nvx * d.nvy * d.V / 2.0
    tot = ax_o[:, 0] + ax_o[:, 1] - 2 * sub
    keep = np.abs(tot) > 0.05 * np.abs(tot).max()
    np.testing.assert_allclose(OBS.axial_ratio(ax_e, d, p.ne)[keep], eo.ref_axial_ratio()[keep],
                               atol=1e-8 if path == BEC_PATH_FP64_PLAIN else 1e-3)
    obs = eng.observables(0, mom[-1, 0])
    assert obs["visibility_scan"] == pytest.approx(eo.ref_visibility(), abs=1e-9 if path == BEC_PATH_FP64_PLAIN else FP32_VIS)


def test_step_graphs_replay_bit_identical(monkeypatch):
    """Steady steps replayed from captured CUDA graphs give the same bits as launching every kernel
    (mixed grids, a 2D slice on the generic plane pass, samples, a pi pulse, then plain evolution)."""
    groups = [
        rb87_params(N=15000, grid=(8, 8, 64), ne=2, noise=True, seed=1),
        rb87_params(N=40000, grid=(16, 16, 128), ne=1, noise=True, seed=2),
        rb87_params(N=25000, grid=(32, 1, 128), ne=2, noise=True, seed=3),
    ]
    gss = [O.ground_state(copy_params(p, ne=1), max_steps=100)[0] for p in groups]
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("BEC_CUDA_GRAPHS", flag)
        eng = Engine(groups, path=BEC_PATH_FP32_BATCHED)
        for g, gs in enumerate(gss):
            eng.init_group(g, gs)
        eng.start_evolution()
        mom = eng.run(100, sample_every=25, pi_pulse_step=50)
        eng.evolve(37)
        out[flag] = (mom, eng.moments(), [eng.get_state(g, t) for g, p in enumerate(groups) for t in range(p.ne)],
                     eng.step_graphs, eng.step_index)
        eng.close()
    on, off = out["1"], out["0"]
    assert on[3] == 2 and off[3] == 0
    assert on[4] == off[4] >= 137
    np.testing.assert_array_equal(on[0], off[0])
    np.testing.assert_array_equal(on[1], off[1])
    for a, b in zip(on[2], off[2]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("path", PATHS)
def test_evolve_and_run_agree(path):
    p = rb87_params(N=30000, grid=(8, 8, 64), ne=1, noise=True, seed=3)
    gs, _ = O.ground_state(copy_params(p, ne=1), max_steps=100)
    m1, e1 = engine_sequence(p, gs, 30, 10, path, use_run=True)
    m2, e2 = engine_sequence(p, gs, 30, 10, path, use_run=False)
    np.testing.assert_allclose(m1, m2, rtol=1e-5 if path else 1e-12)


@pytest.mark.parametrize("path", PATHS)
def test_state_roundtrip(path):
    p = rb87_params(N=30000, grid=(16, 16, 128), ne=2)
    d = O.derive(p)
    rng = np.random.default_rng(0)
    ab = rng.standard_normal((2, d.cells)) + 1j * rng.standard_normal((2, d.cells))
    eng = Engine([p], path=path)
    eng.init_group(0, np.zeros(d.cells))
    eng.set_state(0, 1, ab)
    back = eng.get_state(0, 1)
    assert rel_state_err(back, ab) < (1e-14 if path == BEC_PATH_FP64_PLAIN else 1e-6)


def test_paths_agree_on_16x16x128_ensemble_visibility():
    """A 16x16x128 ensemble of 4 trajectories with noise, 250 steps: ensemble
    visibility of the batched FP32 path within 1e-3 of the FP64 oracle."""
    p = ensemble_16x16x128()
    gs, _ = O.ground_state(copy_params(p, ne=1), max_steps=400)
    mo, eo = oracle_sequence(p, gs, 250, 50)
    me, ee = engine_sequence(p, gs, 250, 50, BEC_PATH_FP32_BATCHED)
    d = eo.d
    err = max(abs(OBS.visibility(a, d, p.ne) - OBS.visibility(b, d, p.ne)) for a, b in zip(me, mo))
    perr = max(abs(OBS.phase(a) - OBS.phase(b)) for a, b in zip(me, mo))
    record("ensemble16_vis", vis_err=err, phase_err=perr)
    assert err < 1e-3
    assert perr < 1e-3
