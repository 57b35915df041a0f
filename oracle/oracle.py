"""ctypes wrapper of the CPU FP64 oracle (oracle/libbec_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline leg, always as the checker or the CPU reference arm,
never as part of the product path.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from bec_b200._abi import (BecDerived, BecGsOpts, BecGsReport, BecMoments, BecParams,
                           BEC_GS_FIXED_STEPS, STATUS_NAMES)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbec_oracle.so")

_lib = None


def build(force=False):
    """Compile libbec_oracle.so with the committed Makefile."""
    if force or not os.path.exists(LIB_PATH) or \
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "bec_oracle.c")):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        dp = P(C.c_double)
        L.oracle_derive.argtypes = [P(BecParams), P(BecDerived)]
        L.oracle_philox4x32_10.argtypes = [P(C.c_uint32), P(C.c_uint32), P(C.c_uint32)]
        L.oracle_philox4x32_10.restype = None
        L.oracle_normals4.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, dp]
        L.oracle_normals4.restype = None
        L.oracle_loss_normals6.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, dp]
        L.oracle_loss_normals6.restype = None
        L.oracle_fft3d.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.oracle_k2_table.argtypes = [P(BecDerived), dp]
        L.oracle_k2_table.restype = None
        L.oracle_potential_table.argtypes = [P(BecDerived), dp]
        L.oracle_potential_table.restype = None
        L.oracle_ground_state.argtypes = [P(BecParams), P(BecGsOpts), dp, P(BecGsReport)]
        L.oracle_gs_measures.argtypes = [P(BecParams), dp, dp, dp, dp, dp]
        L.oracle_create.argtypes = [P(BecParams)]
        L.oracle_create.restype = C.c_void_p
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_free.restype = None
        L.oracle_init.argtypes = [C.c_void_p, dp, dp]
        L.oracle_evolve.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.oracle_pulse.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.oracle_round_fp32.argtypes = [C.c_void_p]
        L.oracle_start_evolution.argtypes = [C.c_void_p, C.c_int]
        L.oracle_moments.argtypes = [C.c_void_p, P(BecMoments)]
        L.oracle_traj_moments.argtypes = [C.c_void_p, P(BecMoments)]
        L.oracle_axial.argtypes = [C.c_void_p, dp]
        L.oracle_get_state.argtypes = [C.c_void_p, C.c_int, dp]
        L.oracle_set_state.argtypes = [C.c_void_p, C.c_int, dp]
        L.oracle_step_index.argtypes = [C.c_void_p]
        L.oracle_step_index.restype = C.c_longlong
        L.oracle_time.argtypes = [C.c_void_p]
        L.oracle_time.restype = C.c_double
        L.oracle_ref_rotated_sums.argtypes = [C.c_void_p, C.c_double, dp, dp]
        L.oracle_ref_visibility.argtypes = [C.c_void_p, dp]
        L.oracle_ref_axial_ratio.argtypes = [C.c_void_p, dp]
        _lib = L
    return _lib


def _check(st, what):
    if st != 0:
        raise RuntimeError(f"oracle {what} failed: {STATUS_NAMES.get(st, st)}")


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def derive(p):
    d = BecDerived()
    _check(lib().oracle_derive(C.byref(p), C.byref(d)), "derive")
    return d


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().oracle_philox4x32_10(c, k, o)
    return list(o)


def loss_normals6(seed, traj, step, cell):
    o = np.zeros(6)
    lib().oracle_loss_normals6(seed, traj, step, cell, _dptr(o))
    return o


def normals4(seed, traj, step, cell, tag):
    o = np.zeros(4)
    lib().oracle_normals4(seed, traj, step, cell, tag, _dptr(o))
    return o


def fft3d(a, sign):
    """Unnormalised 3D DFT of a complex array shaped (nz, ny, nx); sign -1 forward."""
    a = np.ascontiguousarray(a, dtype=np.complex128).copy()
    nz, ny, nx = a.shape
    _check(lib().oracle_fft3d(_dptr(a.view(np.float64)), nx, ny, nz, sign), "fft3d")
    return a


def k2_table(d):
    out = np.zeros(d.cells)
    lib().oracle_k2_table(C.byref(d), _dptr(out))
    return out


def potential_table(d):
    out = np.zeros(d.cells)
    lib().oracle_potential_table(C.byref(d), _dptr(out))
    return out


def ground_state(p, mode=BEC_GS_FIXED_STEPS, max_steps=100, tol=1e-6, check_every=1, warm_start=None,
                 res_tol=0.0):
    d = derive(p)
    o = BecGsOpts()
    o.mode, o.max_steps, o.check_every, o.tol, o.res_tol = mode, max_steps, check_every, tol, res_tol
    ws = None
    if warm_start is not None:
        ws = np.ascontiguousarray(warm_start, dtype=np.complex128)
        o.warm_start = _dptr(ws.view(np.float64))
    psi = np.zeros(d.cells, dtype=np.complex128)
    rep = BecGsReport()
    _check(lib().oracle_ground_state(C.byref(p), C.byref(o), _dptr(psi.view(np.float64)), C.byref(rep)),
           "ground_state")
    return psi, rep


def gs_measures(p, psi):
    psi = np.ascontiguousarray(psi, dtype=np.complex128)
    mu, e, r, n = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    _check(lib().oracle_gs_measures(C.byref(p), _dptr(psi.view(np.float64)), C.byref(mu), C.byref(e),
                                    C.byref(r), C.byref(n)), "gs_measures")
    return mu.value, e.value, r.value, n.value


class OracleEnsemble:
    """One ensemble (ne trajectories) on the CPU, state in the reference's k-space."""

    def __init__(self, p):
        self.p = p
        self.d = derive(p)
        self._h = lib().oracle_create(C.byref(p))
        if not self._h:
            raise RuntimeError("oracle_create failed")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_free(self._h)
            self._h = None

    def init(self, psi_gs, noise=None):
        g = np.ascontiguousarray(psi_gs, dtype=np.complex128)
        nz = None
        if noise is not None:
            nz = np.ascontiguousarray(noise, dtype=np.complex128)
        _check(lib().oracle_init(self._h, _dptr(g.view(np.float64)),
                                 _dptr(nz.view(np.float64)) if nz is not None else None), "init")

    def evolve(self, n, threads=0):
        _check(lib().oracle_evolve(self._h, n, threads), "evolve")

    def pulse(self, theta, phi=0.0):
        _check(lib().oracle_pulse(self._h, theta, phi), "pulse")

    def round_fp32(self):
        """Rounds the stored state to FP32 and back (a rounding-size perturbation)."""
        _check(lib().oracle_round_fp32(self._h), "round_fp32")

    def start_evolution(self, threads=0):
        _check(lib().oracle_start_evolution(self._h, threads), "start_evolution")

    def moments(self):
        m = BecMoments()
        _check(lib().oracle_moments(self._h, C.byref(m)), "moments")
        return np.array([m.t, m.na, m.nb, m.s_re, m.s_im])

    def traj_moments(self):
        ms = (BecMoments * self.d.ne)()
        _check(lib().oracle_traj_moments(self._h, ms), "traj_moments")
        return np.array([[m.t, m.na, m.nb, m.s_re, m.s_im] for m in ms])

    def axial(self):
        out = np.zeros((self.d.nvz, 4))
        _check(lib().oracle_axial(self._h, _dptr(out)), "axial")
        return out

    def get_state(self, traj):
        ab = np.zeros(2 * self.d.cells, dtype=np.complex128)
        _check(lib().oracle_get_state(self._h, traj, _dptr(ab.view(np.float64))), "get_state")
        return ab.reshape(2, self.d.cells)

    def set_state(self, traj, ab):
        ab = np.ascontiguousarray(ab, dtype=np.complex128).reshape(-1)
        _check(lib().oracle_set_state(self._h, traj, _dptr(ab.view(np.float64))), "set_state")

    @property
    def step_index(self):
        return lib().oracle_step_index(self._h)

    @property
    def time(self):
        return lib().oracle_time(self._h)

    def ref_rotated_sums(self, alpha):
        a, b = C.c_double(), C.c_double()
        _check(lib().oracle_ref_rotated_sums(self._h, alpha, C.byref(a), C.byref(b)), "rotated_sums")
        return a.value, b.value

    def ref_visibility(self):
        v = C.c_double()
        _check(lib().oracle_ref_visibility(self._h, C.byref(v)), "visibility")
        return v.value

    def ref_axial_ratio(self):
        out = np.zeros(self.d.nvz)
        _check(lib().oracle_ref_axial_ratio(self._h, _dptr(out)), "axial_ratio")
        return out
