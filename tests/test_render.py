"""Headless projection rendering: BMP round trip and the colour ramp (CPU); the
device projections against projections of the oracle's x-space states (GPU)."""
import numpy as np
import pytest

from bec_b200 import render as R


def test_bmp_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    rgba = rng.uniform(0, 0.999, (5, 7, 4))
    p = tmp_path / "x.bmp"
    R.write_bmp(str(p), rgba)
    back = R.read_bmp(str(p))
    np.testing.assert_array_equal(back, (rgba[..., :3] * 256).astype(np.uint8))


def test_ramp_endpoints_and_midpoints():
    c = R.ramp(np.array([0.0, 1.0 / 3, 2.0 / 3, 1.0]))
    np.testing.assert_allclose(c[0], [0, 0, 255 / 256], atol=1e-9)        # blue
    np.testing.assert_allclose(c[1], [255 / 256] * 3, atol=2 / 256)       # white
    np.testing.assert_allclose(c[2], [255 / 256, 255 / 256, 0], atol=2 / 256)   # yellow
    np.testing.assert_allclose(c[3], [255 / 256, 0, 0], atol=2 / 256)     # red


@pytest.mark.gpu
def test_device_projections_match_oracle():
    from bec_b200.configs import copy_params, rb87_params
    from bec_b200.engine import BEC_PATH_FP32_BATCHED, Engine
    from oracle import oracle as O
    p = rb87_params(N=30000, grid=(16, 16, 128), ne=2, noise=True, seed=7)
    gs, _ = O.ground_state(copy_params(p, ne=1), max_steps=200)
    eng = Engine([p], path=BEC_PATH_FP32_BATCHED)
    eng.init_group(0, gs)
    eng.start_evolution()
    eng.evolve(40)
    img = eng.render_projections(0)
    e = O.OracleEnsemble(p)
    e.init(gs)
    e.start_evolution()
    e.evolve(40)
    d = e.d
    sub = d.V / (2 * d.dV)
    xy = np.zeros((2, d.nvy, d.nvx))
    zy = np.zeros((2, d.nvy, d.nvz))
    for t in range(p.ne):
        a, b = e.get_state(t)
        a = a.reshape(d.nvz, d.nvy, d.nvx)
        b = b.reshape(d.nvz, d.nvy, d.nvx)
        pa = np.abs(a - 1j * b) ** 2 / 2 - sub
        pb = np.abs(-1j * a + b) ** 2 / 2 - sub
        xy[0] += pa.sum(axis=0)
        xy[1] += pb.sum(axis=0)
        zy[0] += pa.sum(axis=2).T
        zy[1] += pb.sum(axis=2).T
    scale = np.abs(xy).max()
    np.testing.assert_allclose(img["levels_xy"], xy, atol=2e-4 * scale)
    np.testing.assert_allclose(img["levels_zy"], zy, atol=2e-4 * np.abs(zy).max())
    mx = 3 * p.N * p.ne / (d.cells * d.dV) * d.nvz
    np.testing.assert_allclose(img["xy_a"][..., :3], R.ramp(img["levels_xy"][0] / mx), atol=2e-3)
