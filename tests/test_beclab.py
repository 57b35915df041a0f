"""The beclab-style front-end (bec_b200/beclab.py): experiment YAML in, `xy` result YAML out.

The reference's front-end is an empty submodule; its only trace is the result files it wrote,
data/gpu_sp_30k.yaml:1-39 and data/experiment_30k.yaml: `xarray` / `yarray` as quoted Python list
strings, `xname`, `yname`, `name`, `description`, `source`, `format: xy`, `ymin` / `ymax`, and
`experimental` in the experiment files. The host-side parts (parameters from an experiment, curves in
that schema, reading them back) run without a GPU; one small experiment runs end to end on the GPU.
"""
import ast
import os

import numpy as np
import pytest
import yaml

from bec_b200 import beclab as B
from bec_b200._abi import BecParams
from bec_b200.configs import rb87_params

# the keys of the reference's xy files (data/gpu_sp_30k.yaml, data/experiment_30k.yaml)
XY_KEYS = {"xarray", "xname", "yarray", "yname", "name", "description", "source", "format", "ymin", "ymax",
           "experimental"}

EXPERIMENT = """
name: 20k atoms, echo
N: 20000
grid: [8, 8, 64]
ensembles: 2
noise: true
fx: 95.0
fy: 95.0
fz: 12.1
a12: 97.5
gamma22: 8.0e-20
seed: 17
dt_evo: 4.0e-5
evolution_time: 0.008
sample_every: 0.002
echo_time: 0.004
phase_points: 8
ground_state: {mode: fixed, max_steps: 80}
"""


def _fields(p):
    return {f: getattr(p, f) for f, _ in BecParams._fields_}


def test_experiment_yaml_round_trips_to_the_same_params(tmp_path):
    f = tmp_path / "ex.yaml"
    f.write_text(EXPERIMENT)
    ex = B.load_yaml(str(f))
    p = B.params_from_experiment(ex)
    expect = rb87_params(N=20000, grid=(8, 8, 64), ne=2, noise=True, seed=17, fx=95.0, fy=95.0, fz=12.1,
                         a12=97.5)
    expect.gamma22 = 8.0e-20
    assert _fields(p) == _fields(expect)
    # dumping the parsed experiment and reading it again gives the same parameters
    g = tmp_path / "ex2.yaml"
    g.write_text(yaml.safe_dump(ex))
    assert _fields(B.params_from_experiment(B.load_yaml(str(g)))) == _fields(p)
    # defaults are the reference's Rb-87 values (wigner.cpp:43-98, SI loss rates)
    assert _fields(B.params_from_experiment({})) == _fields(rb87_params())


def test_xy_curve_schema_and_round_trip(tmp_path):
    t = np.linspace(0.0, 0.6, 61)
    v = np.cos(3 * t) ** 2
    curve = B.xy_dict(t, v, "Time, s", "Visibility", "30k atoms", "GPU (B200), FP32 batched", ymin=0.0, ymax=1.0)
    assert set(curve) == XY_KEYS
    assert curve["format"] == "xy" and curve["experimental"] is False
    path = tmp_path / "visibility.yaml"
    B.write_xy(str(path), curve)
    raw = yaml.safe_load(path.read_text())
    assert isinstance(raw["xarray"], str) and isinstance(raw["yarray"], str)   # quoted list strings
    np.testing.assert_array_equal(ast.literal_eval(raw["xarray"]), t)
    x, y, meta = B.read_xy(str(path))
    np.testing.assert_array_equal(x, t)
    np.testing.assert_array_equal(y, v)
    assert meta["ymin"] == 0.0 and meta["ymax"] == 1.0 and meta["name"] == "30k atoms"


def test_reads_a_file_in_the_reference_layout(tmp_path):
    """A file written the way the reference's data/*.yaml are (folded quoted list strings)."""
    text = ("xarray: '[0.0, 0.0099999999999999915, 0.020000000000000233,\n  0.030000000000000582]'\n"
            "xname: Time, s\nyarray: '[1.0, 0.99, 0.98,\n  0.97]'\nymax: 1.0\nymin: 0.0\nyname: Visibility\n"
            "description: GPU, single precision, 16x16x128, 40mus timestep\nformat: xy\nname: test curve\n"
            "source: 0000000000000000000000000000000000000000\n")
    f = tmp_path / "ref_layout.yaml"
    f.write_text(text)
    x, y, meta = B.read_xy(str(f))
    np.testing.assert_allclose(x, [0.0, 0.01, 0.02, 0.03], atol=1e-15)
    np.testing.assert_allclose(y, [1.0, 0.99, 0.98, 0.97])
    assert meta["format"] == "xy" and set(meta) <= XY_KEYS


@pytest.mark.gpu
def test_experiment_end_to_end_writes_xy_curves(tmp_path):
    f = tmp_path / "ex.yaml"
    f.write_text(EXPERIMENT)
    out = tmp_path / "out"
    B.main([str(f), "--out", str(out)])
    files = sorted(os.listdir(out))
    assert files == ["phase.yaml", "population.yaml", "visibility.yaml"]
    n_samples = 1 + int(round(0.008 / 0.002))
    for name in files:
        x, y, meta = B.read_xy(str(out / name))
        assert set(meta) <= XY_KEYS and meta["format"] == "xy" and meta["name"] == "20k atoms, echo"
        assert len(x) == len(y) == n_samples
        np.testing.assert_allclose(x, np.arange(n_samples) * 0.002, atol=1e-12)
        assert np.isfinite(y).all()
    _, vis, _ = B.read_xy(str(out / "visibility.yaml"))
    # the Wigner estimate of a 2-trajectory ensemble scatters around the true visibility, so it may pass 1
    assert vis[0] == pytest.approx(1.0, abs=1e-2) and (vis < 1.02).all() and (vis > 0.5).all()
    _, pop, _ = B.read_xy(str(out / "population.yaml"))
    assert pop[0] == pytest.approx(20000, rel=0.02) and pop[-1] < pop[0]      # losses remove atoms
    res = B.run_experiment(B.load_yaml(str(f)))
    assert res["phase_scan"].shape == (8, 2) and res["axial_ratio"].shape == (n_samples - 1, 64)
