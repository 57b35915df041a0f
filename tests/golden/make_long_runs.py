"""Generates the long-run oracle fixtures of tests/test_gpu_long_runs.py.

Both runs are the CPU FP64 oracle (oracle/bec_oracle.c) on seeded inputs, so
the fixtures are reproducible bit for bit on any machine with the same libm:

  ensemble_16x16x128_5000.npz  the 3D truncated-Wigner ensemble run: 16x16x128,
      N = 30000, 4 trajectories, Philox vacuum noise keyed by (seed 0,
      trajectory), loss noise on; ground state by 2000 fixed imaginary-time
      steps; one equilibration step, pi/2, then 200 ms (5000 steps of 40 us),
      moments sampled every 250 steps, axial profiles every 1250 steps.
  spin_echo_32x32x256_4traj.npz  the Ramsey / spin-echo sequence at a reduced
      trajectory count: 32x32x256, N = 70000, 4 trajectories, noise and losses
      on; pi/2, 0.5 s (12500 steps), pi, 0.5 s (12500 steps); moments every 500
      steps, axial profiles every 2500 steps; at the end the final pi/2 about
      50 axis angles alpha_j = 2 pi j / 50, evaluated literally
      (halfPiRotate + reduce, wigner_kernel.cu:344-360, wigner.cu:257-265).
  spin_echo_32x32x256_4traj_fp32round.npz  the same run with the stored state rounded to FP32 after
      every step: how far FP32 rounding alone moves this configuration's trajectories and ensemble
      observables (at N = 70000 the trajectories part within about 2000 steps).

    python tests/golden/make_long_runs.py [--only ensemble|spin_echo|spin_echo_fp32round] [--threads N]

Each spin echo takes about an hour of four host cores.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

GS_STEPS = 2000
N_PHASE = 50


def _run(p, steps, sample_every, axial_every, pi_pulse_step, threads, log, round_fp32=False):
    from bec_b200._abi import BEC_GS_FIXED_STEPS
    from bec_b200.configs import copy_params
    from oracle import oracle as O

    t0 = time.time()
    gs, rep = O.ground_state(copy_params(p, ne=1), mode=BEC_GS_FIXED_STEPS, max_steps=GS_STEPS)
    log(f"ground state: {rep.steps} steps, mu {rep.mu:.6f}, {time.time() - t0:.0f} s")
    e = O.OracleEnsemble(p)
    e.init(gs)
    e.start_evolution(threads)
    mom, traj, axial, axial_steps = [], [], [], []
    for i in range(1, steps + 1):
        e.evolve(1, threads)
        if round_fp32:
            e.round_fp32()
        if i % sample_every == 0:
            mom.append(e.moments())
            traj.append(e.traj_moments())
            if i % axial_every == 0:
                axial.append(e.axial())
                axial_steps.append(i)
        if i == pi_pulse_step:
            e.pulse(np.pi, 0.0)
        if i % 1000 == 0:
            log(f"step {i}/{steps}, {time.time() - t0:.0f} s")
    alpha = 2.0 * np.pi * np.arange(N_PHASE) / N_PHASE
    rot = np.array([e.ref_rotated_sums(a) for a in alpha])
    return dict(gs_mu=rep.mu, moments=np.array(mom), traj_moments=np.array(traj), axial=np.array(axial),
                axial_steps=np.array(axial_steps), alpha=alpha, rotated_sums=rot,
                ref_visibility=e.ref_visibility(), ref_axial_ratio=e.ref_axial_ratio(),
                seconds=time.time() - t0)


def ensemble(threads, log):
    from bec_b200.configs import ensemble_16x16x128
    p = ensemble_16x16x128(ne=4, seed=0)
    meta = dict(params="ensemble_16x16x128(ne=4, seed=0)", gs_steps=GS_STEPS, steps=5000, sample_every=250,
                axial_every=1250, pi_pulse_step=-1)
    out = _run(p, 5000, 250, 1250, -1, threads, log)
    return "ensemble_16x16x128_5000.npz", meta, out


def spin_echo(threads, log):
    from bec_b200.configs import spin_echo_32x32x256
    p = spin_echo_32x32x256(ne=4, seed=4)
    meta = dict(params="spin_echo_32x32x256(ne=4, seed=4)", gs_steps=GS_STEPS, steps=25000, sample_every=500,
                axial_every=2500, pi_pulse_step=12500)
    out = _run(p, 25000, 500, 2500, 12500, threads, log)
    return "spin_echo_32x32x256_4traj.npz", meta, out


def spin_echo_fp32round(threads, log):
    from bec_b200.configs import spin_echo_32x32x256
    p = spin_echo_32x32x256(ne=4, seed=4)
    meta = dict(params="spin_echo_32x32x256(ne=4, seed=4)", gs_steps=GS_STEPS, steps=25000, sample_every=500,
                axial_every=2500, pi_pulse_step=12500, perturbation="state rounded to FP32 after every step")
    out = _run(p, 25000, 500, 2500, 12500, threads, log, round_fp32=True)
    return "spin_echo_32x32x256_4traj_fp32round.npz", meta, out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["ensemble", "spin_echo", "spin_echo_fp32round"], default=None)
    ap.add_argument("--threads", type=int, default=4)
    a = ap.parse_args()
    from oracle import oracle as O
    O.build()
    for fn in (ensemble, spin_echo, spin_echo_fp32round):
        if a.only and fn.__name__ != a.only:
            continue
        name, meta, out = fn(a.threads, lambda m: print(f"[{fn.__name__}] {m}", flush=True))
        meta["oracle_seconds"] = out.pop("seconds")
        np.savez_compressed(os.path.join(HERE, name), meta=json.dumps(meta), **out)
        print("wrote", os.path.join(HERE, name), flush=True)


if __name__ == "__main__":
    main()
