"""NN warm start for imaginary-time ground states (the learned part; no reference counterpart).

Pipeline, all on the GPU through the C ABI:
  1. sample parameter sets (N, trap frequencies, scattering lengths) of the
     warm-start workload: N ~ U[5000, 100000], fx = fy and fz each scaled by
     U[0.9, 1.1], a11, a12, a22 each scaled by U[0.98, 1.02], grid 32x32x256;
  2. compute their ground states with the batched FP32 imaginary-time loop
     (mu stopping rule) and keep only the least-squares coefficients of the
     64-term correction over Thomas-Fermi (bec_ground_state_coeffs);
  3. train the MLP 6 -> 256 -> 256 -> 256 -> 64 (BF16 tensor-core GEMMs, FP32
     accumulation, Adam) to map normalised parameters to normalised coefficients;
  4. on held-out parameter sets, run the ground-state loop from Thomas-Fermi
     (cold) and from the network's prediction (warm) with the same stopping rule,
     and compare iterations and device seconds.
The network only seeds the loop; the loop and its |d mu|/mu rule decide.
"""
import ctypes as C
import time

import numpy as np

from ._abi import BEC_GS_MU, BecGsOpts, BecGsReport
from .configs import A11, A12, A22, FX, FY, FZ, rb87_params
from .engine import BEC_PATH_FP32_BATCHED, MLP, Engine, lib

GRID = (32, 32, 256)
WIDTHS = [6, 256, 256, 256, 64]
N_RANGE = (5000.0, 100000.0)


def sample_params(n, seed, grid=GRID):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        N = float(rng.uniform(*N_RANGE))
        sx, sz = rng.uniform(0.9, 1.1, 2)
        s11, s12, s22 = rng.uniform(0.98, 1.02, 3)
        out.append(rb87_params(N=N, grid=grid, ne=1, noise=False, fx=FX * sx, fy=FY * sx, fz=FZ * sz,
                               a11=A11 * s11, a12=A12 * s12, a22=A22 * s22))
    return out


def features(params):
    """Normalised network inputs in [-1, 1]: log N, fx, fz, a11, a12, a22."""
    lo, hi = np.log(N_RANGE[0]), np.log(N_RANGE[1])
    f = []
    for p in params:
        f.append([2 * (np.log(p.N) - lo) / (hi - lo) - 1,
                  (p.fx / FX - 1) / 0.1, (p.fz / FZ - 1) / 0.1,
                  (p.a11 / A11 - 1) / 0.02, (p.a12 / A12 - 1) / 0.02, (p.a22 / A22 - 1) / 0.02])
    return np.array(f, dtype=np.float32)


def ground_states(params, coef_in=None, tol=1e-6, check_every=20, max_steps=40000, chunk=512):
    """Batched ground states; returns (coefficients n x 64, steps, converged, mu, residual, device seconds)."""
    nb = int(lib().bec_warmstart_basis_size())
    n = len(params)
    coef = np.zeros((n, nb))
    steps = np.zeros(n, dtype=np.int64)
    conv = np.zeros(n, dtype=bool)
    mu = np.zeros(n)
    res = np.zeros(n)
    seconds = 0.0
    for a in range(0, n, chunk):
        part = params[a:a + chunk]
        m = len(part)
        eng = Engine(part, path=BEC_PATH_FP32_BATCHED)
        o = BecGsOpts()
        o.mode, o.max_steps, o.check_every, o.tol = BEC_GS_MU, max_steps, check_every, tol
        idx = (C.c_int32 * m)(*range(m))
        cout = np.zeros((m, nb))
        reps = (BecGsReport * m)()
        cin = None
        if coef_in is not None:
            cin = np.ascontiguousarray(coef_in[a:a + m], dtype=np.float64)
        st = lib().bec_ground_state_coeffs(eng._h, m, idx, C.byref(o),
                                           cin.ctypes.data_as(C.POINTER(C.c_double)) if cin is not None else None,
                                           cout.ctypes.data_as(C.POINTER(C.c_double)), reps)
        eng._check(st, "bec_ground_state_coeffs")
        coef[a:a + m] = cout
        for k, r in enumerate(reps):
            steps[a + k], conv[a + k], mu[a + k], res[a + k] = r.steps, bool(r.converged), r.mu, r.residual
        seconds += reps[0].seconds
        eng.close()
    return coef, steps, conv, mu, res, seconds


class WarmStart:
    """Trained network plus the coefficient normalisation."""

    def __init__(self, net, mean, std):
        self.net, self.mean, self.std = net, mean, std

    def predict(self, params):
        y = self.net.forward(features(params))
        return y.astype(np.float64) * self.std + self.mean


def train(params, coef, steps=3000, batch=256, lr=1e-3, seed=0):
    mean = coef.mean(axis=0)
    std = coef.std(axis=0) + 1e-6
    net = MLP(WIDTHS, seed=seed)
    hist = net.train(features(params), ((coef - mean) / std).astype(np.float32), steps=steps, batch=batch, lr=lr,
                     seed=seed)
    return WarmStart(net, mean, std), hist


def run(n_train=4096, n_eval=256, seed=3, train_steps=3000, tol=1e-6, check_every=20, log=print):
    """The full pipeline; returns a dict of measured results."""
    t0 = time.time()
    tr = sample_params(n_train, seed)
    ev = sample_params(n_eval, seed + 1)
    c_tr, s_tr, conv_tr, _, _, sec_tr = ground_states(tr, tol=tol, check_every=check_every)
    log(f"training ground states: {n_train}, converged {conv_tr.mean():.3f}, mean steps {s_tr.mean():.0f}, "
        f"{sec_tr:.1f} device s")
    ws, hist = train(tr, c_tr, steps=train_steps)
    log(f"training loss {hist[:10].mean():.4f} -> {hist[-10:].mean():.5f}")
    c_cold, s_cold, conv_cold, mu_cold, res_cold, sec_cold = ground_states(ev, tol=tol, check_every=check_every)
    pred = ws.predict(ev)
    c_warm, s_warm, conv_warm, mu_warm, res_warm, sec_warm = ground_states(ev, coef_in=pred, tol=tol,
                                                                         check_every=check_every)
    rel_coef_err = np.linalg.norm(pred - c_cold) / np.linalg.norm(c_cold - ws.mean)
    out = {
        "n_train": n_train, "n_eval": n_eval, "train_steps": train_steps,
        "train_loss_first": float(hist[:10].mean()), "train_loss_last": float(hist[-10:].mean()),
        "cold_steps_mean": float(s_cold.mean()), "warm_steps_mean": float(s_warm.mean()),
        "cold_seconds": sec_cold, "warm_seconds": sec_warm,
        "speedup_steps": float(s_cold.mean() / max(s_warm.mean(), 1)),
        "speedup_seconds": float(sec_cold / max(sec_warm, 1e-9)),
        "cold_converged": float(conv_cold.mean()), "warm_converged": float(conv_warm.mean()),
        "mu_rel_diff_max": float(np.max(np.abs(mu_warm - mu_cold) / mu_cold)),
        "residual_warm_max": float(res_warm.max()), "residual_cold_max": float(res_cold.max()),
        "coef_rel_err": float(rel_coef_err), "wall_s": time.time() - t0,
    }
    log(out)
    return out
