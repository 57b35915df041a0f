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
    assert err["visibility"] < 2e-4                   # the stated FP32 visibility bound is 1e-3
    assert err["N1"] < 5e-4 and err["N2"] < 5e-4
    assert err["traj_population"] < 5e-4
    assert err["phase"] < 1e-3
    assert err["phase_noise"] < 1e-3
    assert err["axial_ratio"] < 3e-2


def _ensemble_obs(mom, traj, axial, d, ne):
    """Per-sample ensemble observables of a run: N1, N2, visibility, phase, phase noise (circular spread of the
    per-trajectory phases), and per axial sample the ratio (a - b)/(a + b)(z)."""
    n1, n2 = OBS.populations(mom.T, d, ne)
    vis = np.array([OBS.visibility(m, d, ne) for m in mom])
    phase = np.array([OBS.phase(m) for m in mom])
    noise = np.array([_phase_spread(t) for t in traj])
    ratio = np.array([OBS.axial_ratio(a, d, ne) for a in axial])
    return dict(N1=n1, N2=n2, visibility=vis, phase=phase, phase_noise=noise, axial_ratio=ratio)


def _deviation(x, y, name):
    """max over samples of |x - y| (phases compared on the circle)"""
    if name == "phase":
        return float(np.max(np.abs(np.angle(np.exp(1j * (x - y))))))
    return float(np.max(np.abs(x - y)))


def test_spin_echo_32x32x256_one_second():
    """The trajectories of the FP32 run part from the FP64 oracle's within ~1500 steps: at N = 70000 the
    dynamics amplify any rounding-size difference about a hundredfold per 500 steps, which the oracle
    shows on itself (its run with the stored state rounded to FP32 after every step, the second fixture,
    parts from the unrounded one the same way). So each trajectory is compared over the first 1000 steps,
    and each ensemble observable over the whole second against the FP64 oracle's own deviation under
    FP32 rounding: the FP32 run may differ from the oracle by at most 3 x as much as the rounded oracle run
    does (plus a floor of 1e-3 of the observable's scale)."""
    meta, fx = _load("spin_echo_32x32x256_4traj.npz")
    _, fr = _load("spin_echo_32x32x256_4traj_fp32round.npz")
    p = spin_echo_32x32x256(ne=4, seed=4)
    eng, rep, mom, traj, axial = _engine_run(p, meta)
    assert rep.mu == pytest.approx(float(fx["gs_mu"]), rel=1e-10)
    _compare("long_spin_echo_32x32x256", p, meta, fx, eng, mom, traj, axial)
    d = eng.derived[0]
    ne = p.ne
    # per trajectory, early: samples after 500 and 1000 steps
    to = fx["traj_moments"]
    early = np.abs(traj[:2, :, 1:3] - to[:2, :, 1:3]) / to[:2, :, 1:3]
    assert early.max() < 2e-4
    # ensemble observables against the oracle's deviation under FP32 rounding
    e = _ensemble_obs(mom, traj, axial, d, ne)
    o = _ensemble_obs(fx["moments"], fx["traj_moments"], fx["axial"], d, ne)
    r = _ensemble_obs(fr["moments"], fr["traj_moments"], fr["axial"], d, ne)
    scale = dict(N1=o["N1"].max(), N2=o["N1"].max(), visibility=1.0, phase=np.pi, phase_noise=np.pi, axial_ratio=1.0)
    sub = ne * d.nvx * d.nvy * d.V / 2.0
    keep = [np.abs(a[:, 0] + a[:, 1] - 2 * sub) > 0.2 * np.abs(a[:, 0] + a[:, 1] - 2 * sub).max() for a in fx["axial"]]
    out = {"early_traj_population": float(early.max())}
    for name in ("N1", "N2", "visibility", "phase", "phase_noise", "axial_ratio"):
        if name == "axial_ratio":
            dev_e = max(float(np.abs(x - y)[k].max()) for x, y, k in zip(e[name], o[name], keep))
            dev_r = max(float(np.abs(x - y)[k].max()) for x, y, k in zip(r[name], o[name], keep))
        else:
            dev_e, dev_r = _deviation(e[name], o[name], name), _deviation(r[name], o[name], name)
        out[name] = dev_e
        out[name + "_rounded_oracle"] = dev_r
        assert dev_e <= 3.0 * dev_r + 1e-3 * scale[name], (name, dev_e, dev_r)
    # final pi/2 at 50 phase points: closed form from the FP32 run's moments against the oracle's literal
    # rotation of its own state, against the same for the rounded oracle run
    scan = eng.phase_scan(0, mom[-1], fx["alpha"]) * ne
    dev_scan = float(np.max(np.abs(scan - fx["rotated_sums"])) / np.abs(fx["rotated_sums"]).max())
    dev_scan_r = float(np.max(np.abs(fr["rotated_sums"] - fx["rotated_sums"])) / np.abs(fx["rotated_sums"]).max())
    out["phase_scan"], out["phase_scan_rounded_oracle"] = dev_scan, dev_scan_r
    record("long_spin_echo_vs_rounded_oracle", **out)
    assert dev_scan <= 3.0 * dev_scan_r + 1e-3
