"""bec_init_groups through the C ABI: many ensembles initialised in one call.

The batched call must give the same initial states, bit for bit, as bec_init_group called
once per group: the same per-cell arithmetic runs in one kernel and one preparation pass per
run of consecutive trajectories instead of one pair per group. A complex64 ground state that
is the complex128 one rounded to FP32 gives the same states too, because the FP32 path
rounds the ground state to FP32 on the device either way; so does a real FP32 ground state
(BEC_HOST_R32) of a real profile.
"""
import numpy as np
import pytest

from bec_b200.configs import rb87_params
from bec_b200.engine import BEC_PATH_FP32_BATCHED, BEC_PATH_FP64_PLAIN, BecError, Engine

pytestmark = pytest.mark.gpu


def thomas_fermi(d):
    x = -d.xmax + d.dx * np.arange(d.nvx)
    y = (-d.ymax + d.dy * np.arange(d.nvy)) if d.nvy > 1 else np.zeros(1)
    z = -d.zmax + d.dz * np.arange(d.nvz)
    V = (x[None, None, :] ** 2 + y[None, :, None] ** 2 + z[:, None, None] ** 2 / d.lambda_ ** 2) / 2
    return np.sqrt(np.maximum(d.mu - V, 0.0) / d.g11).reshape(-1).astype(np.complex128)


def mixed_groups():
    """Ensembles of several sizes on three grid classes, a 2D slice among them."""
    out = []
    for i, (grid, ne) in enumerate([((8, 8, 64), 3), ((16, 16, 128), 1), ((8, 8, 64), 1), ((32, 1, 128), 2),
                                    ((16, 16, 128), 2), ((8, 8, 64), 2), ((32, 1, 128), 1), ((16, 16, 128), 1)]):
        out.append(rb87_params(N=12000.0 + 5000.0 * i, grid=grid, ne=ne, noise=True, seed=101 + i))
    return out


def states_of(eng, groups):
    return [eng.get_state(g, t) for g, p in enumerate(groups) for t in range(p.ne)]


def run(init, path=BEC_PATH_FP32_BATCHED, groups=None, steps=6):
    groups = groups or mixed_groups()
    eng = Engine(groups, path=path)
    gs = [thomas_fermi(d) for d in eng.derived]
    init(eng, gs)
    first = states_of(eng, groups)
    eng.start_evolution()
    eng.evolve(steps)
    last = states_of(eng, groups)
    eng.close()
    return first, last


def per_group(eng, gs):
    for g, a in enumerate(gs):
        eng.init_group(g, a)


def assert_same(x, y):
    for part_x, part_y in zip(x, y):
        for a, b in zip(part_x, part_y):
            np.testing.assert_array_equal(a, b)


def test_batched_init_bit_identical():
    ref = run(per_group)
    assert_same(ref, run(lambda eng, gs: eng.init_groups(range(len(gs)), gs)))
    # reversed order of the list, complex64 ground states rounded from the complex128 ones
    assert_same(ref, run(lambda eng, gs: eng.init_groups(list(range(len(gs)))[::-1],
                                                         [a.astype(np.complex64) for a in gs[::-1]])))
    # ground states back to back in one host buffer: consecutive groups arrive in one copy
    assert_same(ref, run(lambda eng, gs: eng.init_groups(range(len(gs)), contiguous_views(gs, np.complex64))))
    assert_same(ref, run(lambda eng, gs: eng.init_groups(range(len(gs)), contiguous_views(gs, np.complex128))))
    # real FP32 ground states (BEC_HOST_R32): the Thomas-Fermi profiles are real, so the same states
    assert_same(ref, run(lambda eng, gs: eng.init_groups(range(len(gs)), contiguous_views(
        [a.real for a in gs], np.float32))))


def contiguous_views(arrays, dtype):
    buf = np.concatenate([a.astype(dtype) for a in arrays])
    out, o = [], 0
    for a in arrays:
        out.append(buf[o:o + a.size])
        o += a.size
    return out


def test_batched_init_subset():
    """A non-contiguous subset in one call, the rest group by group."""
    ref = run(per_group)

    def split(eng, gs):
        odd = [g for g in range(len(gs)) if g % 2]
        eng.init_groups(odd, [gs[g] for g in odd])
        for g in range(0, len(gs), 2):
            eng.init_group(g, gs[g])

    assert_same(ref, run(split))


def test_batched_init_plain_path():
    groups = [rb87_params(N=20000.0, grid=(8, 8, 64), ne=2, noise=True, seed=7),
              rb87_params(N=30000.0, grid=(8, 8, 64), ne=1, noise=True, seed=8)]
    ref = run(per_group, path=BEC_PATH_FP64_PLAIN, groups=groups, steps=2)
    got = run(lambda eng, gs: eng.init_groups([0, 1], gs), path=BEC_PATH_FP64_PLAIN, groups=groups, steps=2)
    assert_same(ref, got)
    # real FP32 ground states reach the FP64 path as their FP32 values
    r32 = run(lambda eng, gs: eng.init_groups([0, 1], [a.real.astype(np.float32) for a in gs]),
              path=BEC_PATH_FP64_PLAIN, groups=groups, steps=2)
    r64 = run(lambda eng, gs: eng.init_groups([0, 1], [a.real.astype(np.float32).astype(np.complex128) for a in gs]),
              path=BEC_PATH_FP64_PLAIN, groups=groups, steps=2)
    assert_same(r64, r32)


def test_batched_init_rejects_bad_arguments():
    groups = mixed_groups()
    eng = Engine(groups, path=BEC_PATH_FP32_BATCHED)
    gs = [thomas_fermi(d) for d in eng.derived]
    with pytest.raises(BecError):
        eng.init_groups([0, 0], [gs[0], gs[0]])          # repeated group
    with pytest.raises(ValueError):
        eng.init_groups([len(groups)], [gs[0]])         # out of range (checked before the call)
    with pytest.raises(ValueError):
        eng.init_groups([1], [gs[0]])                    # wrong size
    # nothing was initialised by the refused calls
    with pytest.raises(BecError):
        eng.start_evolution()
    eng.init_groups([], [])
    eng.close()
