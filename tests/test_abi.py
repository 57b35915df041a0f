"""The C-ABI boundary without a GPU: the library loads, exports every function
include/bec.h declares, its structures match the ctypes mirror, and its host
parameter derivation equals the oracle's restatement of fillDerivedParameters."""
import ctypes as C
import os
import re
import subprocess
import sys
import tempfile

import pytest

from bec_b200 import _abi
from bec_b200 import engine as E
from bec_b200.configs import slice_2d_32x128, ensemble_16x16x128, uneven_batch, spin_echo_32x32x256, rb87_params
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bec.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bec_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = E.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(E.SIGNATURES), "ctypes signature table out of date"
    assert lib.bec_abi_version() == 3


def test_struct_layout_matches_c_compiler():
    prog = r"""
#include <stdio.h>
#include <stddef.h>
#include "bec.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(bec_params), sizeof(bec_derived), sizeof(bec_gs_opts),
         sizeof(bec_gs_report), sizeof(bec_moments), sizeof(bec_obs), sizeof(bec_schedule));
  printf("%zu %zu %zu\n", offsetof(bec_params, seed), offsetof(bec_derived, n_equil_steps), offsetof(bec_gs_opts, warm_start));
  printf("%zu %zu\n", offsetof(bec_gs_opts, res_tol), offsetof(bec_gs_report, step_residual));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as td:
        src = os.path.join(td, "l.c")
        open(src, "w").write(prog)
        exe = os.path.join(td, "l")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    sizes = [int(v) for v in out]
    expect = [C.sizeof(_abi.BecParams), C.sizeof(_abi.BecDerived), C.sizeof(_abi.BecGsOpts),
              C.sizeof(_abi.BecGsReport), C.sizeof(_abi.BecMoments), C.sizeof(_abi.BecObs),
              C.sizeof(_abi.BecSchedule),
              _abi.BecParams.seed.offset, _abi.BecDerived.n_equil_steps.offset, _abi.BecGsOpts.warm_start.offset,
              _abi.BecGsOpts.res_tol.offset, _abi.BecGsReport.step_residual.offset]
    assert sizes == expect


@pytest.mark.parametrize("params", [slice_2d_32x128(), ensemble_16x16x128(), spin_echo_32x32x256(ne=2)] + uneven_batch(n_traj=6)
                         + [rb87_params(t_equilib=1e-3), rb87_params(grid=(32, 1, 64), fy=50.0)])
def test_product_derivation_equals_oracle(params):
    d1 = E.derive(params)
    d2 = O.derive(params)
    for name, _ in _abi.BecDerived._fields_:
        v1, v2 = getattr(d1, name), getattr(d2, name)
        assert v1 == pytest.approx(v2, rel=1e-15, abs=0), name


@pytest.mark.parametrize("change,status", [
    (dict(nvx=12), _abi.BEC_ERR_UNSUPPORTED_GRID),
    (dict(nvz=1), _abi.BEC_ERR_UNSUPPORTED_GRID),
    (dict(N=0.0), _abi.BEC_ERR_INVALID_ARG),
    (dict(ne=0), _abi.BEC_ERR_INVALID_ARG),
    (dict(itmax=0), _abi.BEC_ERR_INVALID_ARG),
])
def test_invalid_parameters_are_rejected(change, status):
    p = rb87_params()
    for k, v in change.items():
        setattr(p, k, v)
    d = _abi.BecDerived()
    assert E.lib().bec_derive_params(C.byref(p), C.byref(d)) == status


def test_null_arguments_do_not_crash():
    lib = E.lib()
    assert lib.bec_derive_params(None, None) == _abi.BEC_ERR_INVALID_ARG
    assert lib.bec_create(None, 0, 0, None) == _abi.BEC_ERR_INVALID_ARG
    lib.bec_destroy(None)
    assert lib.bec_last_error(None) == b"null context"


def test_create_without_device_fails_cleanly():
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("a GPU is visible")
    p = rb87_params()
    h = C.c_void_p()
    st = E.lib().bec_create(C.byref(p), 1, _abi.BEC_PATH_FP32_BATCHED, C.byref(h))
    assert st == _abi.BEC_ERR_NO_DEVICE
    assert not h.value
    with pytest.raises(E.BecError):
        E.Engine(p)
