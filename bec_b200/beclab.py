"""beclab-style front-end: experiment YAML in, `xy` result YAML out.

The reference's Python front-end (programs/beclab.py, an un-vendored git
submodule) is absent; its only trace is the result files it wrote,
data/gpu_sp_30k.yaml and data/gpu_sp_30k_4ens.yaml: `xy` curves with
`xarray`/`yarray` stored as quoted Python list strings, plus `xname`, `yname`,
`name`, `description`, `source`, `format`, `ymin`/`ymax` and `experimental`.
This module reads an experiment description (the parameter surface of
programs/bec_wigner_3d.cuda/defines.h:25-54 in SI units, plus the Ramsey /
spin-echo schedule), runs it on the engine and writes curves in that schema.

    python -m bec_b200.beclab experiment.yaml --out results/

Experiment keys (all optional, defaults are the reference's Rb-87 values):
  N, grid [nvx, nvy, nvz], a11, a12, a22, m, fx, fy, fz, detuning,
  gamma111, gamma12, gamma22, noise (bool), loss_noise (bool), ensembles,
  itmax, dt_steady, dt_evo, t_equilib, seed, path (fp32 | fp64),
  evolution_time (s), sample_every (s), echo_time (s, pi pulse; null = none),
  ground_state: {mode: fixed | mu | reference, max_steps, tol, check_every},
  phase_points (final pi/2 phase scan points).
"""
import argparse
import os

import numpy as np

from . import observables as OBS
from ._abi import BEC_GS_FIXED_STEPS, BEC_GS_MU, BEC_GS_REFERENCE_E
from .configs import rb87_params
from .engine import BEC_PATH_FP32_BATCHED, BEC_PATH_FP64_PLAIN, Engine

GS_MODES = {"fixed": BEC_GS_FIXED_STEPS, "mu": BEC_GS_MU, "reference": BEC_GS_REFERENCE_E}


def load_yaml(path):
    import yaml
    with open(path) as f:
        return yaml.safe_load(f) or {}


def params_from_experiment(ex):
    """bec_params of one ensemble from an experiment dictionary."""
    grid = tuple(ex.get("grid", (16, 16, 128)))
    noise = bool(ex.get("noise", False))
    p = rb87_params(N=float(ex.get("N", 30000)), grid=grid, ne=int(ex.get("ensembles", 1)), noise=noise,
                    loss_noise=ex.get("loss_noise"), detuning=float(ex.get("detuning", 0.0)),
                    dt_evo=float(ex.get("dt_evo", 4e-5)), dt_steady=float(ex.get("dt_steady", 1e-5)),
                    t_equilib=float(ex.get("t_equilib", 0.0)), itmax=int(ex.get("itmax", 1)),
                    seed=int(ex.get("seed", 0)))
    for k in ("a11", "a12", "a22", "m", "fx", "fy", "fz", "gamma111", "gamma12", "gamma22"):
        if k in ex:
            setattr(p, k, float(ex[k]))
    return p


def steps_for(t, dt):
    """Number of steps of size dt covering time t (rounded to nearest)."""
    return int(round(t / dt))


def run_experiment(ex):
    """Runs one experiment; returns a dict of curves (numpy arrays)."""
    p = params_from_experiment(ex)
    path = BEC_PATH_FP64_PLAIN if str(ex.get("path", "fp32")).lower() == "fp64" else BEC_PATH_FP32_BATCHED
    gs_cfg = ex.get("ground_state", {}) or {}
    with Engine([p], path=path) as eng:
        gs, rep = eng.ground_state(0, mode=GS_MODES[str(gs_cfg.get("mode", "mu"))],
                                   max_steps=int(gs_cfg.get("max_steps", 20000)), tol=float(gs_cfg.get("tol", 1e-7)),
                                   check_every=int(gs_cfg.get("check_every", 10)))
        eng.init_group(0, gs)
        eng.start_evolution()
        n = steps_for(float(ex.get("evolution_time", 0.1)), p.dt_evo)
        every = max(1, steps_for(float(ex.get("sample_every", 0.01)), p.dt_evo))
        echo = ex.get("echo_time")
        pi_step = steps_for(float(echo), p.dt_evo) if echo is not None else -1
        m0 = eng.moments()[0]
        mom, axial = eng.run(n, sample_every=every, pi_pulse_step=pi_step, axial=True)
        d = eng.derived[0]
        rows = [m0] + [m for m in mom[:, 0]]
        t = np.array([r[0] for r in rows])
        vis = np.array([OBS.visibility(r, d, p.ne) for r in rows])
        scan = np.array([OBS.visibility_scan(r, d, p.ne) for r in rows])
        phase = np.array([OBS.phase(r) for r in rows])
        n1 = np.array([OBS.populations(r, d, p.ne)[0] for r in rows])
        n2 = np.array([OBS.populations(r, d, p.ne)[1] for r in rows])
        out = {"t": t, "visibility": vis, "visibility_scan": scan, "phase": phase, "N1": n1, "N2": n2,
               "axial_ratio": np.array([OBS.axial_ratio(a, d, p.ne) for a in axial[0]]),
               "ground_state": {"steps": rep.steps, "mu": rep.mu, "residual": rep.residual}}
        npts = int(ex.get("phase_points", 0))
        if npts > 0:
            alphas = np.linspace(0.0, 2 * np.pi, npts, endpoint=False)
            out["phase_scan"] = eng.phase_scan(0, mom[-1, 0], alphas)
            out["phase_scan_alpha"] = alphas
        return out


def xy_dict(x, y, xname, yname, name, description, source="bec_b200", ymin=None, ymax=None):
    """One curve in the data/*.yaml `xy` schema."""
    d = {"xarray": repr([float(v) for v in x]), "xname": xname,
         "yarray": repr([float(v) for v in y]), "yname": yname,
         "name": name, "description": description, "source": source, "format": "xy",
         "experimental": False}
    if ymin is not None:
        d["ymin"] = ymin
    if ymax is not None:
        d["ymax"] = ymax
    return d


def write_xy(path, curve):
    import yaml
    with open(path, "w") as f:
        yaml.safe_dump(curve, f, default_flow_style=False)


def read_xy(path):
    """(x, y, meta) of an `xy` YAML file such as data/gpu_sp_30k.yaml."""
    import ast
    d = load_yaml(path)
    return np.array(ast.literal_eval(d["xarray"])), np.array(ast.literal_eval(d["yarray"])), d


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("experiment")
    ap.add_argument("--out", default=".")
    a = ap.parse_args(argv)
    ex = load_yaml(a.experiment)
    res = run_experiment(ex)
    os.makedirs(a.out, exist_ok=True)
    label = ex.get("name", f"{int(ex.get('N', 30000)) // 1000}k atoms")
    desc = f"GPU (B200), FP32 batched, {'x'.join(str(v) for v in ex.get('grid', (16, 16, 128)))}, " \
           f"{ex.get('ensembles', 1)} ensembles, {float(ex.get('dt_evo', 4e-5)) * 1e6:.0f}mus timestep"
    write_xy(os.path.join(a.out, "visibility.yaml"),
             xy_dict(res["t"], res["visibility"], "Time, s", "Visibility", label, desc, ymin=0.0, ymax=1.0))
    write_xy(os.path.join(a.out, "population.yaml"),
             xy_dict(res["t"], res["N1"] + res["N2"], "Time, s", "N", label, desc, ymin=0))
    write_xy(os.path.join(a.out, "phase.yaml"), xy_dict(res["t"], res["phase"], "Time, s", "Phase, rad", label, desc))
    print(f"wrote {a.out}/visibility.yaml, population.yaml, phase.yaml")


if __name__ == "__main__":
    main()
