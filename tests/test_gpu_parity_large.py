"""Oracle parity of the 32x32x256 real-time kernels and of a step that runs every fast pass.

The 32x32x256 class carries most of the uneven-batch workload: its plane pass (32x32 planes, line
transforms split over two warps) and its nz = 256 pencil pass. Here they run against the CPU FP64
oracle on the same inputs, with Philox vacuum noise, loss noise and losses on, moments-only samples
(read from the stored state while a half kick is pending), a pi pulse fused into the next pencil pass,
and a sample with axial profiles (the observing pass that ends a step); propagate,
programs/bec_wigner_3d.cuda/wigner.cu:178-199, with wigner_kernel.cu:137-151 and :184-229.

Tolerances are those of the FP32 batched path in test_gpu_parity.py: per-trajectory states within
2e-4 of the oracle's max |psi| (<= 200 steps), moments within 1e-4 relative.
"""
import numpy as np
import pytest

from bec_b200 import observables as OBS
from bec_b200._abi import BEC_GS_FIXED_STEPS
from bec_b200.configs import copy_params, rb87_params
from bec_b200.engine import BEC_PATH_FP32_BATCHED, BEC_PATH_FP64_PLAIN, Engine
from oracle import oracle as O
from parity_util import moments_rel_err, record, rel_state_err

pytestmark = pytest.mark.gpu

FP32_STATE = 2e-4
FP32_MOM = 1e-4


def _gpu_ground_state(p, steps):
    """x-space ground state from the FP64 plain path (1e-10 of the oracle's), used as the common input."""
    eng = Engine([copy_params(p, ne=1)], path=BEC_PATH_FP64_PLAIN)
    psi, rep = eng.ground_state(0, mode=BEC_GS_FIXED_STEPS, max_steps=steps)
    eng.close()
    assert rep.steps == steps
    return psi


def test_32x32x256_noise_losses_pulse_samples():
    """2 trajectories, N = 70000: pi/2, 100 steps with moments-only samples every 50 and a pi pulse
    after step 75, then 50 steps ending in a sample with axial profiles."""
    p = rb87_params(N=70000, grid=(32, 32, 256), ne=2, noise=True, seed=21)
    gs = _gpu_ground_state(p, 200)

    eng = Engine([p], path=BEC_PATH_FP32_BATCHED)
    eng.init_group(0, gs)
    eng.start_evolution()
    m1 = eng.run(100, sample_every=50, pi_pulse_step=75)[:, 0, :]
    m2, ax = eng.run(50, sample_every=50, axial=True)
    m2 = m2[:, 0, :]

    e = O.OracleEnsemble(p)
    e.init(gs)
    e.start_evolution()
    mo = []
    for i in range(1, 151):
        e.evolve(1)
        if i % 50 == 0:
            mo.append(e.moments())
        if i == 75:
            e.pulse(np.pi, 0.0)
    me = np.concatenate([m1, m2])
    assert me.shape == (3, 5)
    np.testing.assert_allclose(me[:, 0], np.array(mo)[:, 0], rtol=1e-12)
    mom_err = max(max(moments_rel_err(a, b)) for a, b in zip(me, mo))
    st_err = max(rel_state_err(eng.get_state(0, t), e.get_state(t)) for t in range(p.ne))
    tm_e, tm_o = eng.traj_moments(), e.traj_moments()
    tm_err = float(np.max(np.abs(tm_e[:, 1:3] - tm_o[:, 1:3]) / tm_o[:, 1:3]))

    ax_o, ax_e = e.axial(), ax[0][-1]
    d = e.d
    sub = p.ne * d.nvx * d.nvy * d.V / 2.0
    tot = ax_o[:, 0] + ax_o[:, 1] - 2 * sub
    keep = np.abs(tot) > 0.05 * np.abs(tot).max()
    ratio_err = float(np.abs(OBS.axial_ratio(ax_e, d, p.ne)[keep] - e.ref_axial_ratio()[keep]).max())
    ax_err = float(np.abs(ax_e[:, :2] - ax_o[:, :2]).max() / ax_o[:, :2].max())
    vis_err = abs(OBS.visibility(me[-1], d, p.ne) - OBS.visibility(mo[-1], d, p.ne))
    record("parity_32x32x256", state_err=st_err, moments_err=mom_err, traj_mom_err=tm_err, axial_err=ax_err,
           axial_ratio_err=ratio_err, vis_err=vis_err)
    assert st_err < FP32_STATE
    assert mom_err < FP32_MOM
    assert tm_err < FP32_MOM
    assert ax_err < 10 * FP32_MOM
    assert ratio_err < 1e-3
    assert vis_err < 1e-4


def test_mixed_classes_in_one_captured_step():
    """8x8x64, 16x16x128 and 32x32x256 ensembles in one context: every steady step replays a captured
    graph that runs the three register plane passes and the three register pencil passes."""
    groups = [
        rb87_params(N=15000, grid=(8, 8, 64), ne=2, noise=True, seed=31, fx=92.0, fy=92.0),
        rb87_params(N=40000, grid=(16, 16, 128), ne=1, noise=True, seed=32, fz=12.5),
        rb87_params(N=60000, grid=(32, 32, 256), ne=1, noise=True, seed=33, fx=101.0, fy=101.0),
    ]
    eng = Engine(groups, path=BEC_PATH_FP32_BATCHED)
    ens = []
    for g, p in enumerate(groups):
        gs = _gpu_ground_state(p, 150)
        eng.init_group(g, gs)
        e = O.OracleEnsemble(p)
        e.init(gs)
        e.start_evolution()
        ens.append(e)
    eng.start_evolution()
    eng.evolve(45)                     # one eager step, then 8-step and 1-step graph replays
    assert eng.step_graphs == 2
    mom = eng.moments()
    worst_s, worst_m = 0.0, 0.0
    for g, (p, e) in enumerate(zip(groups, ens)):
        e.evolve(45)
        worst_m = max(worst_m, max(moments_rel_err(mom[g], e.moments())))
        for t in range(p.ne):
            worst_s = max(worst_s, rel_state_err(eng.get_state(g, t), e.get_state(t)))
    record("parity_mixed_classes_graphs", state_err=worst_s, moments_err=worst_m)
    assert worst_s < FP32_STATE
    assert worst_m < FP32_MOM
