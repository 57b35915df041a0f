"""ctypes binding of libbec.so (include/bec.h).

This is the Python face of the engine: `Engine` owns a bec_ctx and mirrors the
reference's host entry points (programs/bec_wigner_3d.cuda/wigner.cpp:32-40):
calculateSteadyState -> ground_state, initEvolution -> init_group +
start_evolution, calculateEvolution -> evolve / run, plus observables.

There is no CPU fallback: if the CUDA library cannot be loaded or no device
is visible, construction raises.
"""
import ctypes as C
import os

import numpy as np

from ._abi import (BecDerived, BecGsOpts, BecGsReport, BecMoments, BecObs, BecParams, BecSchedule,
                   BEC_GS_FIXED_STEPS, BEC_HOST_C128, BEC_HOST_C64, BEC_HOST_R32, BEC_LR_CONSTANT, BEC_PATH_FP32_BATCHED, BEC_PATH_FP64_PLAIN, STATUS_NAMES)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbec.so")

_lib = None

# every function of include/bec.h: name -> (restype, argtypes)
_P = C.POINTER
_dp = _P(C.c_double)
SIGNATURES = {
    "bec_abi_version": (C.c_int32, []),
    "bec_derive_params": (C.c_int, [_P(BecParams), _P(BecDerived)]),
    "bec_create": (C.c_int, [_P(BecParams), C.c_int32, C.c_int32, _P(C.c_void_p)]),
    "bec_destroy": (None, [C.c_void_p]),
    "bec_last_error": (C.c_char_p, [C.c_void_p]),
    "bec_group_info": (C.c_int, [C.c_void_p, C.c_int32, _P(BecDerived)]),
    "bec_total_trajectories": (C.c_int64, [C.c_void_p]),
    "bec_ground_state": (C.c_int, [C.c_void_p, C.c_int32, _P(BecGsOpts), _dp, _P(BecGsReport)]),
    "bec_ground_state_batch": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_int32), _P(BecGsOpts), _P(_dp),
                                         _P(BecGsReport)]),
    "bec_init_group": (C.c_int, [C.c_void_p, C.c_int32, _dp, _dp]),
    "bec_init_groups": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_int32), _P(C.c_void_p), C.c_int32]),
    "bec_evolve": (C.c_int, [C.c_void_p, C.c_int32]),
    "bec_pulse": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "bec_start_evolution": (C.c_int, [C.c_void_p]),
    "bec_moments_now": (C.c_int, [C.c_void_p, _P(BecMoments)]),
    "bec_axial_now": (C.c_int, [C.c_void_p, C.c_int32, _dp]),
    "bec_traj_moments_now": (C.c_int, [C.c_void_p, _P(BecMoments)]),
    "bec_run": (C.c_int, [C.c_void_p, _P(BecSchedule), _P(BecMoments), _dp]),
    "bec_observables": (C.c_int, [C.c_void_p, C.c_int32, _P(BecMoments), _P(BecObs)]),
    "bec_phase_scan": (C.c_int, [C.c_void_p, C.c_int32, _P(BecMoments), C.c_int32, _dp, _dp]),
    "bec_get_state": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, _dp]),
    "bec_set_state": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, _dp]),
    "bec_step_index": (C.c_int64, [C.c_void_p]),
    "bec_evolution_steps": (C.c_int64, [C.c_void_p]),
    "bec_set_step_index": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64]),
    "bec_checkpoint_bytes": (C.c_int64, [C.c_void_p]),
    "bec_checkpoint_save": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    "bec_checkpoint_load": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    "bec_step_graphs": (C.c_int32, [C.c_void_p]),
    "bec_step_plan": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32]),
    "bec_profile_fused_step": (C.c_int, [C.c_void_p, C.c_int32, _dp, _P(C.c_int64)]),
    "bec_last_device_ms": (C.c_double, [C.c_void_p]),
    "bec_last_launch_count": (C.c_int64, [C.c_void_p]),
    "bec_profile_steps": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, _P(C.c_int32), _P(C.c_int64), _dp,
                                    _P(C.c_int32)]),
    "bec_moments_device_noalloc": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_void_p,
                                             C.c_void_p]),
    "bec_ground_state_coeffs": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_int32), _P(BecGsOpts), _dp, _dp,
                                          _P(C.c_float), _P(BecGsReport)]),
    "bec_warmstart_basis_size": (C.c_int32, []),
    "bec_warmstart_set_basis": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                          _P(C.c_float)]),
    "bec_pulse_finite": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
    "bec_render_projections": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_float), _P(C.c_float), _P(C.c_float),
                                         _P(C.c_float), _P(C.c_float), _P(C.c_float)]),
    "bec_mlp_create": (C.c_int, [_P(C.c_int32), C.c_int32, C.c_uint64, _P(C.c_void_p)]),
    "bec_mlp_destroy": (None, [C.c_void_p]),
    "bec_mlp_param_count": (C.c_int64, [C.c_void_p]),
    "bec_mlp_get_params": (C.c_int, [C.c_void_p, _P(C.c_float)]),
    "bec_mlp_set_params": (C.c_int, [C.c_void_p, _P(C.c_float)]),
    "bec_mlp_forward": (C.c_int, [C.c_void_p, _P(C.c_float), C.c_int32, _P(C.c_float)]),
    "bec_mlp_gradients": (C.c_int, [C.c_void_p, _P(C.c_float), _P(C.c_float), C.c_int32, _P(C.c_float),
                                    _P(C.c_float)]),
    "bec_mlp_train": (C.c_int, [C.c_void_p, _P(C.c_float), _P(C.c_float), C.c_int32, C.c_int32, C.c_int32,
                                C.c_float, C.c_int32, C.c_uint64, _P(C.c_float)]),
}


class BecError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib():
    """Loads libbec.so (building it first if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build
            build.build()
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _dptr(a):
    return a.ctypes.data_as(_dp)


def derive(p):
    d = BecDerived()
    st = lib().bec_derive_params(C.byref(p), C.byref(d))
    if st:
        raise BecError(st, "bec_derive_params")
    return d


class Engine:
    """A bec_ctx: one or more ensembles ("groups") on the current CUDA device."""

    def __init__(self, groups, path=BEC_PATH_FP32_BATCHED):
        if isinstance(groups, BecParams):
            groups = [groups]
        self.params = list(groups)
        arr = (BecParams * len(self.params))(*self.params)
        h = C.c_void_p()
        st = lib().bec_create(arr, len(self.params), path, C.byref(h))
        if st:
            raise BecError(st, "bec_create")
        self._h = h
        self.path = path
        self.derived = [self._info(g) for g in range(len(self.params))]

    def close(self):
        if getattr(self, "_h", None):
            lib().bec_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st, what):
        if st:
            raise BecError(st, f"{what}: {lib().bec_last_error(self._h).decode()}")

    def _info(self, g):
        d = BecDerived()
        self._check(lib().bec_group_info(self._h, g, C.byref(d)), "bec_group_info")
        return d

    @property
    def n_groups(self):
        return len(self.params)

    @property
    def n_traj(self):
        return int(lib().bec_total_trajectories(self._h))

    @property
    def step_index(self):
        return int(lib().bec_step_index(self._h))

    @property
    def evolution_steps(self):
        return int(lib().bec_evolution_steps(self._h))

    def set_step_index(self, step, evolution_steps):
        """Continues the Philox loss-noise stream of a saved run (after set_state in a fresh context)."""
        self._check(lib().bec_set_step_index(self._h, int(step), int(evolution_steps)), "bec_set_step_index")

    def checkpoint(self):
        """The whole evolution state, bit for bit, as bytes (bec_checkpoint_save)."""
        n = int(lib().bec_checkpoint_bytes(self._h))
        buf = C.create_string_buffer(n)
        self._check(lib().bec_checkpoint_save(self._h, buf, n), "bec_checkpoint_save")
        return buf.raw

    def restore(self, blob):
        """Loads a checkpoint of a context with the same groups and path (bec_checkpoint_load)."""
        buf = C.create_string_buffer(bytes(blob), len(blob))
        self._check(lib().bec_checkpoint_load(self._h, buf, len(blob)), "bec_checkpoint_load")

    @property
    def step_plan(self):
        """The split-step schedule (bec_step_plan) as a dict."""
        import json
        buf = C.create_string_buffer(4096)
        self._check(lib().bec_step_plan(self._h, buf, len(buf)), "bec_step_plan")
        return json.loads(buf.value.decode())

    @property
    def step_graphs(self):
        return int(lib().bec_step_graphs(self._h))

    @property
    def last_device_ms(self):
        return float(lib().bec_last_device_ms(self._h))

    @property
    def last_launch_count(self):
        return int(lib().bec_last_launch_count(self._h))

    # ---- ground state (calculateSteadyState, wigner.cu:84-175)
    def ground_state(self, group=0, mode=BEC_GS_FIXED_STEPS, max_steps=100, tol=1e-6, check_every=1,
                     warm_start=None, res_tol=0.0):
        d = self.derived[group]
        o = BecGsOpts()
        o.mode, o.max_steps, o.check_every, o.tol, o.res_tol = mode, max_steps, check_every, tol, res_tol
        ws = None
        if warm_start is not None:
            ws = np.ascontiguousarray(warm_start, dtype=np.complex128).reshape(-1)
            if ws.size != d.cells:
                raise ValueError("warm start size")
            o.warm_start = _dptr(ws.view(np.float64))
        psi = np.zeros(d.cells, dtype=np.complex128)
        rep = BecGsReport()
        self._check(lib().bec_ground_state(self._h, group, C.byref(o), _dptr(psi.view(np.float64)),
                                           C.byref(rep)), "bec_ground_state")
        return psi, rep

    # ---- ensembles (initEvolution, wigner.cu:202-227)
    def init_group(self, group, psi_gs, noise=None):
        d = self.derived[group]
        g = np.ascontiguousarray(psi_gs, dtype=np.complex128).reshape(-1)
        if g.size != d.cells:
            raise ValueError("ground-state size")
        nz = None
        if noise is not None:
            nz = np.ascontiguousarray(noise, dtype=np.complex128).reshape(-1)
            if nz.size != 2 * d.cells * self.params[group].ne:
                raise ValueError("noise size")
        self._check(lib().bec_init_group(self._h, group, _dptr(g.view(np.float64)),
                                         _dptr(nz.view(np.float64)) if nz is not None else None),
                    "bec_init_group")

    def init_groups(self, groups, psi_gs):
        """bec_init_groups: initialise many groups in one call (vacuum noise from Philox).

        psi_gs[i] is the ground state of groups[i]; complex64 arrays are passed as complex64
        (half the host-to-device bytes), float32 arrays as real FP32 ground states (a quarter),
        anything else as complex128. Pinned arrays copy fastest."""
        groups = [int(g) for g in groups]
        if len(groups) != len(psi_gs):
            raise ValueError("one ground state per group")
        c64 = len(psi_gs) > 0 and all(np.asarray(a).dtype == np.complex64 for a in psi_gs)
        r32 = len(psi_gs) > 0 and all(np.asarray(a).dtype == np.float32 for a in psi_gs)
        dt = np.complex64 if c64 else np.float32 if r32 else np.complex128
        arrs = []
        for g, a in zip(groups, psi_gs):
            a = np.ascontiguousarray(a, dtype=dt).reshape(-1)
            if not 0 <= g < self.n_groups:
                raise ValueError("group index out of range")
            if a.size != self.derived[g].cells:
                raise ValueError("ground-state size")
            arrs.append(a)
        n = len(groups)
        gi = (C.c_int32 * max(n, 1))(*groups)
        ptrs = (C.c_void_p * max(n, 1))(*[a.ctypes.data for a in arrs])
        self._check(lib().bec_init_groups(self._h, n, gi, ptrs,
                                          BEC_HOST_C64 if c64 else BEC_HOST_R32 if r32 else BEC_HOST_C128),
                    "bec_init_groups")

    def start_evolution(self):
        self._check(lib().bec_start_evolution(self._h), "bec_start_evolution")

    def evolve(self, n):
        self._check(lib().bec_evolve(self._h, int(n)), "bec_evolve")

    def pulse(self, theta, phi=0.0):
        self._check(lib().bec_pulse(self._h, float(theta), float(phi)), "bec_pulse")

    def pulse_finite(self, rabi_hz, duration_s, phi=0.0):
        """Rabi pulse of finite duration (coupling on during round(duration/dt) split steps)."""
        self._check(lib().bec_pulse_finite(self._h, float(rabi_hz), float(duration_s), float(phi)),
                    "bec_pulse_finite")

    # ---- observables
    def moments(self):
        ms = (BecMoments * self.n_groups)()
        self._check(lib().bec_moments_now(self._h, ms), "bec_moments_now")
        return np.array([[m.t, m.na, m.nb, m.s_re, m.s_im] for m in ms])

    def traj_moments(self):
        ms = (BecMoments * self.n_traj)()
        self._check(lib().bec_traj_moments_now(self._h, ms), "bec_traj_moments_now")
        return np.array([[m.t, m.na, m.nb, m.s_re, m.s_im] for m in ms])

    def axial(self, group=0):
        out = np.zeros((self.derived[group].nvz, 4))
        self._check(lib().bec_axial_now(self._h, group, _dptr(out)), "bec_axial_now")
        return out

    def observables(self, group, moments_row):
        m = BecMoments(*[float(v) for v in moments_row])
        o = BecObs()
        self._check(lib().bec_observables(self._h, group, C.byref(m), C.byref(o)), "bec_observables")
        return {k: getattr(o, k) for k, _ in BecObs._fields_}

    def phase_scan(self, group, moments_row, alphas):
        m = BecMoments(*[float(v) for v in moments_row])
        al = np.ascontiguousarray(alphas, dtype=np.float64)
        out = np.zeros(2 * al.size)
        self._check(lib().bec_phase_scan(self._h, group, C.byref(m), al.size, _dptr(al), _dptr(out)),
                    "bec_phase_scan")
        return out.reshape(-1, 2)

    def run(self, n_steps, sample_every=0, pi_pulse_step=-1, axial=False):
        """Runs n_steps, returning moments [n_samples, n_groups, 5] (and axial profiles)."""
        s = BecSchedule(int(n_steps), int(sample_every), int(pi_pulse_step), int(bool(axial)))
        every = sample_every if sample_every > 0 else max(n_steps, 1)
        n_samples = n_steps // every
        ms = (BecMoments * max(n_samples * self.n_groups, 1))()
        ax = None
        if axial:
            ax = np.zeros(max(n_samples, 1) * sum(4 * d.nvz for d in self.derived))
        self._check(lib().bec_run(self._h, C.byref(s), ms, _dptr(ax) if ax is not None else None), "bec_run")
        mom = np.array([[m.t, m.na, m.nb, m.s_re, m.s_im] for m in ms][: n_samples * self.n_groups])
        mom = mom.reshape(n_samples, self.n_groups, 5)
        if axial:
            out, off = [], 0
            for d in self.derived:
                out.append(ax.reshape(max(n_samples, 1), -1)[:n_samples, off:off + 4 * d.nvz].reshape(n_samples, d.nvz, 4))
                off += 4 * d.nvz
            return mom, out
        return mom

    def render_projections(self, group=0):
        """RGBA images (float, h x w x 4) of the xy and zy projections of both components after a
        pi/2 pulse, plus the projected densities: dict(xy_a, xy_b, zy_a, zy_b, levels_xy, levels_zy)."""
        d = self.derived[group]
        f = lambda *s: np.zeros(s, dtype=np.float32)
        xy_a, xy_b = f(d.nvy, d.nvx, 4), f(d.nvy, d.nvx, 4)
        zy_a, zy_b = f(d.nvy, d.nvz, 4), f(d.nvy, d.nvz, 4)
        lxy, lzy = f(2, d.nvy, d.nvx), f(2, d.nvy, d.nvz)
        p = lambda a: a.ctypes.data_as(_P(C.c_float))
        self._check(lib().bec_render_projections(self._h, group, p(xy_a), p(xy_b), p(zy_a), p(zy_b), p(lxy), p(lzy)),
                    "bec_render_projections")
        return dict(xy_a=xy_a, xy_b=xy_b, zy_a=zy_a, zy_b=zy_b, levels_xy=lxy, levels_zy=lzy)

    # ---- warm-start ground states (coefficients of the correction over Thomas-Fermi)
    def ground_state_coeffs(self, groups=None, mode=BEC_GS_FIXED_STEPS, max_steps=100, tol=1e-6, check_every=20,
                            res_tol=0.0, coef_in=None, want_coef=True, want_profiles=False):
        """Batched FP32 ground states of groups sharing one grid; returns (coef n x 64 or None,
        profiles n x cells float32 or None, reports)."""
        groups = list(range(self.n_groups)) if groups is None else list(groups)
        n = len(groups)
        nb = int(lib().bec_warmstart_basis_size())
        o = BecGsOpts()
        o.mode, o.max_steps, o.check_every, o.tol, o.res_tol = mode, max_steps, check_every, tol, res_tol
        idx = (C.c_int32 * n)(*groups)
        cin = None
        if coef_in is not None:
            cin = np.ascontiguousarray(coef_in, dtype=np.float64).reshape(n, nb)
        cout = np.zeros((n, nb)) if want_coef else None
        prof = np.zeros((n, self.derived[groups[0]].cells), dtype=np.float32) if want_profiles else None
        reps = (BecGsReport * n)()
        self._check(lib().bec_ground_state_coeffs(self._h, n, idx, C.byref(o),
                                                  _dptr(cin) if cin is not None else None,
                                                  _dptr(cout) if cout is not None else None,
                                                  prof.ctypes.data_as(_P(C.c_float)) if prof is not None else None,
                                                  reps), "bec_ground_state_coeffs")
        return cout, prof, list(reps)

    def set_warmstart_basis(self, grid, basis):
        """Installs basis rows (nb x cells float32, nb <= 64) for grid (nvx, nvy, nvz); None removes it."""
        nx, ny, nz = grid
        if basis is None:
            self._check(lib().bec_warmstart_set_basis(self._h, nx, ny, nz, 0, None), "bec_warmstart_set_basis")
            return
        b = np.ascontiguousarray(basis, dtype=np.float32)
        if b.ndim != 2 or b.shape[1] != nx * ny * nz:
            raise ValueError("basis shape")
        self._check(lib().bec_warmstart_set_basis(self._h, nx, ny, nz, b.shape[0], b.ctypes.data_as(_P(C.c_float))),
                    "bec_warmstart_set_basis")

    def profile_fused_step(self, n_steps):
        """(mean ms of one step's fused launch, cells it covers) over n_steps steady steps."""
        ms = C.c_double()
        cells = C.c_int64()
        self._check(lib().bec_profile_fused_step(self._h, int(n_steps), C.byref(ms), C.byref(cells)),
                    "bec_profile_fused_step")
        return ms.value, int(cells.value)

    def profile_steps(self, n_steps, max_classes=16):
        """Per grid class: dict(dims, traj, z_ms, plane_ms) mean device time per launch."""
        dims = (C.c_int32 * (3 * max_classes))()
        traj = (C.c_int64 * max_classes)()
        ms = (C.c_double * (2 * max_classes))()
        nc = C.c_int32()
        self._check(lib().bec_profile_steps(self._h, int(n_steps), max_classes, dims, traj, ms, C.byref(nc)),
                    "bec_profile_steps")
        return [dict(dims=tuple(dims[3 * c:3 * c + 3]), traj=int(traj[c]), z_ms=ms[2 * c], plane_ms=ms[2 * c + 1])
                for c in range(min(nc.value, max_classes))]

    # ---- state I/O (checkpoint / parity)
    def get_state(self, group, traj):
        d = self.derived[group]
        ab = np.zeros(2 * d.cells, dtype=np.complex128)
        self._check(lib().bec_get_state(self._h, group, traj, _dptr(ab.view(np.float64))), "bec_get_state")
        return ab.reshape(2, d.cells)

    def set_state(self, group, traj, ab):
        ab = np.ascontiguousarray(ab, dtype=np.complex128).reshape(-1)
        self._check(lib().bec_set_state(self._h, group, traj, _dptr(ab.view(np.float64))), "bec_set_state")


def _fptr(a):
    return a.ctypes.data_as(_P(C.c_float))


class MLP:
    """The warm-start network (bec_mlp_*): tanh MLP, tensor-core GEMMs on split BF16 operands, FP32 accumulation."""

    def __init__(self, widths, seed=0):
        self.widths = [int(w) for w in widths]
        arr = (C.c_int32 * len(self.widths))(*self.widths)
        h = C.c_void_p()
        st = lib().bec_mlp_create(arr, len(self.widths) - 1, seed, C.byref(h))
        if st:
            raise BecError(st, "bec_mlp_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().bec_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _check(self, st, what):
        if st:
            raise BecError(st, what)

    @property
    def n_params(self):
        return int(lib().bec_mlp_param_count(self._h))

    def get_params(self):
        p = np.zeros(self.n_params, dtype=np.float32)
        self._check(lib().bec_mlp_get_params(self._h, _fptr(p)), "bec_mlp_get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(lib().bec_mlp_set_params(self._h, _fptr(p)), "bec_mlp_set_params")

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], self.widths[-1]), dtype=np.float32)
        self._check(lib().bec_mlp_forward(self._h, _fptr(x), x.shape[0], _fptr(y)), "bec_mlp_forward")
        return y

    def gradients(self, x, target):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(target, dtype=np.float32)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = C.c_float()
        self._check(lib().bec_mlp_gradients(self._h, _fptr(x), _fptr(t), x.shape[0], C.byref(loss), _fptr(g)),
                    "bec_mlp_gradients")
        return float(loss.value), g

    def train(self, x, target, steps, batch=256, lr=1e-3, seed=0, schedule=BEC_LR_CONSTANT):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(target, dtype=np.float32)
        hist = np.zeros(max(steps, 1), dtype=np.float32)
        self._check(lib().bec_mlp_train(self._h, _fptr(x), _fptr(t), x.shape[0], batch, steps, lr, schedule, seed,
                                        _fptr(hist)), "bec_mlp_train")
        return hist[:steps]


__all__ = ["Engine", "MLP", "BecError", "derive", "lib", "BEC_PATH_FP32_BATCHED", "BEC_PATH_FP64_PLAIN"]
