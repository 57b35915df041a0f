"""Generates tests/golden/gpu_sp_30k.json.

1. The reference's stored GPU result data/gpu_sp_30k.yaml ("GPU, single
   precision, 16x16x128, 40mus timestep", 30k atoms, no noise): visibility
   against time, 0 to 0.6 s in 10 ms samples. Read from the reference tree,
   which exists only where this script is run (not on the GPU machine).
2. The CPU FP64 oracle's visibility curve for the same run with the Rb-87
   loss rates of bec_b200.configs (GAMMA*): ground state by the reference's
   own stopping rule (wigner.cu:148-156), one equilibration step, pi/2, then
   15000 steps of 40 us sampled every 250 steps.
3. The same oracle run with the loss rates written in the reference's
   parameter set (SOURCE_GAMMA*, wigner.cpp:74-76), the rates that reproduce
   the stored curve (detuning does not enter the visibility).

    python tests/golden/make_golden.py --reference-data <reference checkout>/data
"""
import argparse
import ast
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-data", required=True,
                    help="the reference's data/ directory (holds gpu_sp_30k.yaml and gpu_sp_30k_4ens.yaml)")
    a = ap.parse_args()
    import yaml
    from bec_b200 import observables as OBS
    from bec_b200._abi import BEC_GS_REFERENCE_E
    from bec_b200.configs import SOURCE_GAMMA111, SOURCE_GAMMA12, SOURCE_GAMMA22, copy_params, rb87_params
    from oracle import oracle as O

    ref = yaml.safe_load(open(os.path.join(a.reference_data, "gpu_sp_30k.yaml")))
    xs = [float(v) for v in ast.literal_eval(ref["xarray"])]
    ys = [float(v) for v in ast.literal_eval(ref["yarray"])]
    ref4 = yaml.safe_load(open(os.path.join(a.reference_data, "gpu_sp_30k_4ens.yaml")))

    def curve(p):
        gs, rep = O.ground_state(p, mode=BEC_GS_REFERENCE_E, max_steps=20000)
        e = O.OracleEnsemble(p)
        e.init(gs)
        e.start_evolution()
        t, vis, scan, mom = [], [], [], []
        for k in range(len(xs)):
            if k:
                e.evolve(250, 0)
            m = e.moments()
            t.append(float(m[0]))
            vis.append(float(OBS.visibility(m, e.d, 1)))
            scan.append(float(OBS.visibility_scan(m, e.d, 1)))
            mom.append([float(v) for v in m])
        return rep.steps, t, vis, scan, mom

    p = rb87_params(N=30000, grid=(16, 16, 128), ne=1, noise=False)
    gs_steps, t, vis, scan, mom = curve(p)
    ps = copy_params(p, gamma111=SOURCE_GAMMA111, gamma12=SOURCE_GAMMA12, gamma22=SOURCE_GAMMA22)
    gs_steps_s, t_s, vis_s, scan_s, mom_s = curve(ps)
    out = {
        "reference": {"file": "data/gpu_sp_30k.yaml", "description": ref["description"], "name": ref["name"],
                      "source": ref["source"], "t": xs, "visibility": ys},
        "reference_4ens": {"file": "data/gpu_sp_30k_4ens.yaml", "description": ref4["description"],
                           "t": [float(v) for v in ast.literal_eval(ref4["xarray"])],
                           "visibility": [float(v) for v in ast.literal_eval(ref4["yarray"])]},
        "oracle": {"params": "rb87_params(N=30000, grid=(16,16,128), ne=1, noise=False) with SI losses",
                   "ground_state_steps": gs_steps, "steps_per_sample": 250, "t": t, "visibility": vis,
                   "visibility_scan": scan, "moments": mom},
        "oracle_source_losses": {"params": "the same with the loss rates of the reference's parameter set "
                                           "(SOURCE_GAMMA111/12/22)",
                                 "ground_state_steps": gs_steps_s, "steps_per_sample": 250, "t": t_s,
                                 "visibility": vis_s, "visibility_scan": scan_s, "moments": mom_s},
    }
    with open(os.path.join(HERE, "gpu_sp_30k.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "gpu_sp_30k.json"))


if __name__ == "__main__":
    main()
