"""Parameter sets of the workloads this engine is measured on.

Physical values are those of the reference's Rb-87 runs
(programs/bec_wigner_3d.cuda/wigner.cpp:43-98): m = 1.443160648e-25 kg,
a11/a12/a22 = 100.40/97.66/95.00 Bohr radii, fx = fy = 97.6 Hz, fz = 11.96 Hz,
itmax = 1, dt_steady = 1e-5 s, dt_evo = 4e-5 s, t_equilib = 0. Loss rates are
SI: gamma111 = 5.4e-42 m^6/s, gamma12 = 1.51e-20 m^3/s, gamma22 = 8.1e-20 m^3/s.
Detuning is 0 Hz unless given (the workloads do not state one).
"""
import numpy as np

from ._abi import BecParams

RB87_MASS = 1.443160648e-25
A11, A12, A22 = 100.40, 97.66, 95.00
FX, FY, FZ = 97.6, 97.6, 11.96
GAMMA111, GAMMA12, GAMMA22 = 5.4e-42, 1.51e-20, 8.1e-20
# The loss rates written, commented out, in the reference's parameter set (wigner.cpp:74-76: 5.4e-30 cm^6/s,
# 0.78e-13 cm^3/s, 1.194e-13 cm^3/s), in SI units. The stored GPU curve data/gpu_sp_30k.yaml (30k atoms, no
# noise) is reproduced with these over its whole 0.6 s, and not with the rates above.
SOURCE_GAMMA111, SOURCE_GAMMA12, SOURCE_GAMMA22 = 5.4e-42, 0.78e-19, 1.194e-19


def rb87_params(N=30000.0, grid=(16, 16, 128), ne=1, noise=False, losses=True,
                loss_noise=None, fx=FX, fy=FY, fz=FZ, a11=A11, a12=A12, a22=A22,
                detuning=0.0, dt_evo=4e-5, dt_steady=1e-5, t_equilib=0.0, itmax=1,
                seed=0):
    """One ensemble of the two-component Rb-87 model.

    grid is (nvx, nvy, nvz); nvy == 1 selects the 2D x-z slice.
    noise turns on the initial vacuum noise (Va = Vb = 1); loss_noise
    (default: equal to noise) adds the Wigner loss-noise terms.
    """
    p = BecParams()
    p.a11, p.a12, p.a22 = a11, a12, a22
    p.m = RB87_MASS
    p.fx, p.fy, p.fz = fx, fy, fz
    p.N = float(N)
    p.detuning = detuning
    if losses:
        p.gamma111, p.gamma12, p.gamma22 = GAMMA111, GAMMA12, GAMMA22
    p.Va = p.Vb = 1.0 if noise else 0.0
    p.nvx, p.nvy, p.nvz = grid
    p.itmax = itmax
    p.dt_steady, p.t_equilib, p.dt_evo = dt_steady, t_equilib, dt_evo
    p.ne = ne
    p.loss_noise = int(noise if loss_noise is None else loss_noise)
    p.seed = seed
    return p


def copy_params(p, **changes):
    q = BecParams()
    C_fields = [f[0] for f in BecParams._fields_]
    for f in C_fields:
        setattr(q, f, getattr(p, f))
    for k, v in changes.items():
        setattr(q, k, v)
    return q


def slice_2d_32x128():
    """2D x-z slice, 32x128, one noise-free trajectory, N = 30000:
    2000 imaginary-time steps, pi/2, 100 ms (2500 steps)."""
    return rb87_params(N=30000, grid=(32, 1, 128), ne=1, noise=False)


def ensemble_16x16x128(ne=4, seed=0):
    """3D truncated Wigner, 16x16x128, 4 trajectories, N = 30000, 200 ms."""
    return rb87_params(N=30000, grid=(16, 16, 128), ne=ne, noise=True, seed=seed)


UNEVEN_GRIDS = ((8, 8, 64), (16, 16, 128), (32, 32, 256))


def uneven_batch(n_traj=1024, seed=2, grids=UNEVEN_GRIDS):
    """Uneven batch: n_traj single-trajectory ensembles, grid drawn uniformly
    from `grids`, N ~ U[5000, 70000], fx and fz each scaled by U[0.9, 1.1]
    (fy follows fx), noise and losses on. Seeded; returns a list of params."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_traj):
        g = grids[int(rng.integers(len(grids)))]
        N = float(rng.uniform(5000.0, 70000.0))
        sx = float(rng.uniform(0.9, 1.1))
        sz = float(rng.uniform(0.9, 1.1))
        out.append(rb87_params(N=N, grid=g, ne=1, noise=True, fx=FX * sx, fy=FY * sx,
                               fz=FZ * sz, seed=1000003 * seed + i))
    return out


def spin_echo_32x32x256(ne=1024, seed=4):
    """Ramsey / spin echo: N = 70000, 32x32x256, 1024 trajectories, 1.0 s with a
    pi pulse at 0.5 s, final pi/2 sampled at 50 phase points."""
    return rb87_params(N=70000, grid=(32, 32, 256), ne=ne, noise=True, seed=seed)
