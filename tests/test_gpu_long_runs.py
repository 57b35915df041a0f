"""Long runs of the batched FP32 path against committed FP64 oracle runs of the same seeds.

Fixtures (tests/golden/make_long_runs.py, the CPU FP64 oracle):
  * the 3D truncated-Wigner ensemble: 16x16x128, N = 30000, 4 trajectories, Philox vacuum and loss
    noise, pi/2, then 200 ms (5000 steps of 40 us), sampled every 250 steps;
  * the Ramsey / spin-echo sequence at 4 trajectories: 32x32x256, N = 70000, pi/2, 0.5 s, pi, 0.5 s
    (25000 steps), sampled every 500 steps, then the final pi/2 about 50 axis angles.
The ground state is the FP64 plain path's (2000 fixed imaginary-time steps, within 1e-10 of the
oracle's), so both runs start from the same input. Per sample the test compares each observable of
the reference's (wigner.cu:257-303, :363-369): per-trajectory populations N1, N2, ensemble visibility,
phase arg <psi1|psi2>, the per-trajectory phase spread (phase noise) and the axial ratio
(a - b)/(a + b)(z) after a pi/2; and, after the spin echo, the populations of the final pi/2 at the
50 phase points against the oracle's literal halfPiRotate + reduce. The measured worst errors are
stated in the design notes; the bounds below leave them a margin.
"""
import json
import os

import numpy as np
import pytest

from bec_b200 import observables as OBS
from bec_b200._abi import BEC_GS_FIXED_STEPS
from bec_b200.configs import copy_params, ensemble_16x16x128, spin_echo_32x32x256
from bec_b200.engine import BEC_PATH_FP32_BATCHED, BEC_PATH_FP64_PLAIN, Engine
from parity_util import dump, record

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    z = np.load(os.path.join(HERE, name))
    meta = json.loads(str(z["meta"]))
    return meta, {k: z[k] for k in z.files if k != "meta"}


def _phase_spread(traj):
    """circular standard deviation of the per-trajectory phases arg s_t"""
    ph = np.arctan2(traj[:, 4], traj[:, 3])
    r = np.abs(np.exp(1j * ph).mean())
    return float(np.sqrt(max(-2.0 * np.log(max(r, 1e-300)), 0.0)))


def _engine_run(p, meta):
    gs_eng = Engine([copy_params(p, ne=1)], path=BEC_PATH_FP64_PLAIN)
    gs, rep = gs_eng.ground_state(0, mode=BEC_GS_FIXED_STEPS, max_steps=meta["gs_steps"])
    gs_eng.close()
    eng = Engine([p], path=BEC_PATH_FP32_BATCHED)
    eng.init_group(0, gs)
    eng.start_evolution()
    every, steps, pi_step = meta["sample_every"], meta["steps"], meta["pi_pulse_step"]
    mom, traj, axial = [], [], []
    done = 0
    # run sample by sample so that per-trajectory moments are read at every sample; axial samples end
    # their step with the observing pass, moments-only samples read the stored state
    while done < steps:
        k = every
        want_axial = (done + k) % meta["axial_every"] == 0
        pulse_at = pi_step - done if done < pi_step <= done + k else -1
        out = eng.run(k, sample_every=k, pi_pulse_step=pulse_at, axial=want_axial)
        if want_axial:
            m, ax = out
            axial.append(ax[0][-1])
        else:
            m = out
        mom.append(m[-1, 0])
        traj.append(eng.traj_moments())
        done += k
    return eng, rep, np.array(mom), np.array(traj), np.array(axial)


def _compare(name, p, meta, fx, eng, mom, traj, axial):
    d = eng.derived[0]
    mo, to, axo = fx["moments"], fx["traj_moments"], fx["axial"]
    assert mom.shape == mo.shape and traj.shape == to.shape and axial.shape == axo.shape
    np.testing.assert_allclose(mom[:, 0], mo[:, 0], rtol=1e-12)
    n1e, n2e = OBS.populations(mom.T, d, p.ne)
    n1o, n2o = OBS.populations(mo.T, d, p.ne)
    err = dict(
        N1=float(np.max(np.abs(n1e - n1o) / n1o.max())),
        N2=float(np.max(np.abs(n2e - n2o) / max(n1o.max(), n2o.max()))),
        visibility=float(max(abs(OBS.visibility(a, d, p.ne) - OBS.visibility(b, d, p.ne)) for a, b in zip(mom, mo))),
        phase=float(max(abs(np.angle(np.exp(1j * (OBS.phase(a) - OBS.phase(b))))) for a, b in zip(mom, mo))),
        phase_noise=float(max(abs(_phase_spread(a) - _phase_spread(b)) for a, b in zip(traj, to))),
        traj_population=float(np.max(np.abs(traj[:, :, 1:3] - to[:, :, 1:3]) / to[:, :, 1:3].max())),
    )
    # (a - b)/(a + b)(z) is a local quantity: differences of FP32 rounding size grow in it by about x7 per
    # 1250 steps (the FP64 oracle itself, its state rounded to FP32 after every step, moves by 6e-4 over
    # 5000 steps), most at the condensate's edges; it is compared where the density is above 20 % of its
    # peak, and at 5 % for the record
    sub = p.ne * d.nvx * d.nvy * d.V / 2.0
    for th, key in ((0.2, "axial_ratio"), (0.05, "axial_ratio_edge")):
        worst = 0.0
        for ae, ao in zip(axial, axo):
            tot = ao[:, 0] + ao[:, 1] - 2 * sub
            keep = np.abs(tot) > th * np.abs(tot).max()
            worst = max(worst, float(np.abs(OBS.axial_ratio(ae, d, p.ne) - OBS.axial_ratio(ao, d, p.ne))[keep].max()))
        err[key] = worst
    record(name, **err)
    dump(name, moments=mom, traj_moments=traj, axial=axial)
    return err


def test_ensemble_16x16x128_200ms():
    meta, fx = _load("ensemble_16x16x128_5000.npz")
    p = ensemble_16x16x128(ne=4, seed=0)
    eng, rep, mom, traj, axial = _engine_run(p, meta)
    assert rep.mu == pytest.approx(float(fx["gs_mu"]), rel=1e-10)
    err = _compare("long_ensemble_16x16x128", p, meta, fx, eng, mom, traj, axial)
    assert err["visibility"] < 2e-4                   # the north-star bound is 1e-3
    assert err["N1"] < 5e-4 and err["N2"] < 5e-4
    assert err["traj_population"] < 5e-4
    assert err["phase"] < 1e-3
    assert err["phase_noise"] < 1e-3
    assert err["axial_ratio"] < 3e-2


def _traj_obs(tm, d):
    """per-trajectory N1, N2, visibility and phase from per-trajectory moments [ne, 5]"""
    n1 = np.array([OBS.populations(r, d, 1)[0] for r in tm])
    n2 = np.array([OBS.populations(r, d, 1)[1] for r in tm])
    vis = np.array([OBS.visibility(r, d, 1) for r in tm])
    ph = np.arctan2(tm[:, 4], tm[:, 3])
    return n1, n2, vis, ph


def test_spin_echo_32x32x256_one_second():
    """Over the full second the trajectories of the two runs part (the dynamics amplify FP32 rounding
    differences exponentially at N = 70000; see the design notes for the FP64 oracle's own sensitivity),
    so each trajectory is compared over the first 1000 steps and the ensemble observables over the whole
    run against their statistical error: 4 x the standard error of a 4-trajectory mean, from the spread
    of the trajectories of both runs."""
    meta, fx = _load("spin_echo_32x32x256_4traj.npz")
    p = spin_echo_32x32x256(ne=4, seed=4)
    eng, rep, mom, traj, axial = _engine_run(p, meta)
    assert rep.mu == pytest.approx(float(fx["gs_mu"]), rel=1e-10)
    err = _compare("long_spin_echo_32x32x256", p, meta, fx, eng, mom, traj, axial)
    d = eng.derived[0]
    to = fx["traj_moments"]
    ne = p.ne
    # per trajectory, early: samples after 500 and 1000 steps
    early = np.abs(traj[:2, :, 1:3] - to[:2, :, 1:3]) / to[:2, :, 1:3]
    record("long_spin_echo_early", traj_population_1000=float(early.max()))
    assert early.max() < 2e-4
    # ensemble observables against their statistical error
    worst = {}
    for k in range(len(mom)):
        oe, oo = _traj_obs(traj[k], d), _traj_obs(to[k], d)
        ens_e = (*OBS.populations(mom[k], d, ne), OBS.visibility(mom[k], d, ne), OBS.phase(mom[k]))
        ens_o = (*OBS.populations(fx["moments"][k], d, ne), OBS.visibility(fx["moments"][k], d, ne),
                 OBS.phase(fx["moments"][k]))
        for name, i in (("N1", 0), ("N2", 1), ("visibility", 2), ("phase", 3)):
            if name == "phase":
                diff = abs(np.angle(np.exp(1j * (ens_e[i] - ens_o[i]))))
                spread = [np.sqrt(max(-2 * np.log(max(abs(np.exp(1j * o[i]).mean()), 1e-300)), 0.0)) for o in (oe, oo)]
            else:
                diff = abs(ens_e[i] - ens_o[i])
                spread = [o[i].std(ddof=1) for o in (oe, oo)]
            sigma = np.sqrt(spread[0] ** 2 + spread[1] ** 2) / np.sqrt(ne)
            worst[name] = max(worst.get(name, 0.0), diff / max(sigma, 1e-12))
    record("long_spin_echo_sigmas", **worst)
    for name, z in worst.items():
        assert z < 4.0, (name, z)
    # final pi/2 at 50 phase points: closed form from the FP32 run's moments against the oracle's literal
    # rotation of its own state, relative to the spread of the trajectories' rotated populations
    scan = eng.phase_scan(0, mom[-1], fx["alpha"]) * ne
    rot = fx["rotated_sums"]
    per_traj = np.array([[OBS.rotated(r, d, 1, a) for a in fx["alpha"]] for r in to[-1]])   # [ne, 50, 2]
    sigma_scan = per_traj.std(axis=0, ddof=1) * np.sqrt(ne) * np.sqrt(2.0)
    z_scan = float(np.max(np.abs(scan - rot) / sigma_scan))
    record("long_spin_echo_phase_scan", phase_scan=float(np.max(np.abs(scan - rot)) / np.abs(rot).max()),
           phase_scan_sigmas=z_scan)
    assert z_scan < 4.0
