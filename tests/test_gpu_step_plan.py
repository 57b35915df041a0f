"""The split-step schedules: per-pass launches (plane passes at 16 or 20 warps per SM; pencil passes on the
register kernel or the persistent TMA kernel, and 8x8x64 steps as one on-chip launch, chosen per grid class) and the
fused step kernel (one persistent launch per split step) on its autotuned work list.

Every schedule computes the same bits: launches per pass and grid class, with any pencil kernel, the
two-phase work list, and the interleaved work lists at every distance, with samples, a pi pulse, captured
step graphs and a grid class that the fused kernel does not take (a 2D slice). The autotuner picks one of
the candidates and reports its timings; a steady step of the fused classes is one launch. A dependency
wait that runs out (a plane item told to wait for one pencil item more than exists), and a TMA tile wait
that runs out (the first tile of every CTA also waiting for a flag that nothing sets), end with
BEC_ERR_CUDA and leave the device usable.
"""
import numpy as np
import pytest

from bec_b200._abi import BEC_ERR_CUDA
from bec_b200.configs import copy_params, rb87_params
from bec_b200.engine import BEC_PATH_FP32_BATCHED, BecError, Engine
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GROUPS = [
    rb87_params(N=15000, grid=(8, 8, 64), ne=3, noise=True, seed=51),
    rb87_params(N=40000, grid=(16, 16, 128), ne=2, noise=True, seed=52),
    rb87_params(N=60000, grid=(32, 32, 256), ne=2, noise=True, seed=53),
    rb87_params(N=25000, grid=(32, 1, 128), ne=2, noise=True, seed=54),
    rb87_params(N=20000, grid=(16, 16, 64), ne=1, noise=True, seed=55),
]


# forced per-pass schedules and their candidate numbers: register pencils at 16 / 20 warps per SM, then every class
# on the TMA pencil kernel
PER_PASS = {"unfused": 0, "unfused-20": 1, "unfused-tma": 2, "unfused-20-tma": 3, "unfused-onchip": 2}
N_PER_PASS = 4
N_CANDIDATES = N_PER_PASS + 5


@pytest.fixture(scope="module")
def ground_states():
    return [O.ground_state(copy_params(p, ne=1), max_steps=20)[0] for p in GROUPS]


def _run(monkeypatch, plan, gss, groups=GROUPS):
    if plan is None:
        monkeypatch.delenv("BEC_STEP_PLAN", raising=False)
    else:
        monkeypatch.setenv("BEC_STEP_PLAN", plan)
    eng = Engine(groups, path=BEC_PATH_FP32_BATCHED)
    for g, gs in enumerate(gss):
        eng.init_group(g, gs)
    eng.start_evolution()
    mom = eng.run(60, sample_every=20, pi_pulse_step=30)
    eng.evolve(17)
    out = dict(mom=mom, now=eng.moments(), plan=eng.step_plan,
               states=[eng.get_state(g, t) for g, p in enumerate(groups) for t in range(p.ne)])
    eng.close()
    return out


def test_every_schedule_gives_the_same_bits(monkeypatch, ground_states):
    ref = _run(monkeypatch, "unfused", ground_states)
    assert ref["plan"]["candidate"] == 0 and ref["plan"]["fused_classes"] == 0
    for plan in list(PER_PASS)[1:] + ["0", "1", "2", "3", "4", None]:
        got = _run(monkeypatch, plan, ground_states)
        p = got["plan"]
        if plan is None:
            assert p["chosen"] in ("autotuned", "cached") and 0 <= p["candidate"] < N_CANDIDATES
        elif plan in PER_PASS:
            assert p["chosen"] == "forced" and p["candidate"] == PER_PASS[plan]
            want = "tma" if plan.endswith("tma") else "register"
            assert all(k["kernel"] == want for k in p["pencil_kernels"])
            # "unfused-onchip": the 8x8x64 class's steady steps as one launch with its state in shared memory
            assert all(k["onchip"] == (plan == "unfused-onchip" and k["grid"] == [8, 8, 64]) for k in p["pencil_kernels"])
        else:
            assert p["chosen"] == "forced" and p["candidate"] == int(plan) + N_PER_PASS
        # the fused kernel takes every class but the 2D slice
        assert p["fused_classes"] == (4 if p["candidate"] >= N_PER_PASS else 0)
        np.testing.assert_array_equal(got["mom"], ref["mom"])
        np.testing.assert_array_equal(got["now"], ref["now"])
        for a, b in zip(got["states"], ref["states"]):
            np.testing.assert_array_equal(a, b)


def _three_classes(ground_states):
    groups = [GROUPS[0], GROUPS[1], GROUPS[2]]
    eng = Engine(groups, path=BEC_PATH_FP32_BATCHED)
    for g in range(3):
        eng.init_group(g, ground_states[g])
    eng.start_evolution()
    eng.evolve(3)
    return eng, groups


def test_autotuner_reports_timings(monkeypatch, ground_states):
    monkeypatch.delenv("BEC_STEP_PLAN", raising=False)
    eng, _ = _three_classes(ground_states)
    p = eng.step_plan
    assert p["chosen"] in ("autotuned", "cached")
    assert len(p["candidates"]) == N_CANDIDATES
    if p["chosen"] == "autotuned":
        ms = p["candidate_ms_per_step"]           # the four per-pass schedules, the work lists 0..4
        assert len(ms) == N_CANDIDATES and all(v > 0 for v in ms)
        assert ms[p["candidate"]] == min(ms)
        # per grid class, both pencil kernels were timed, and the tuned schedules use the faster; an 8x8x64
        # class also timed its on-chip step against its pencil plus plane launches
        for k in p["pencil_kernels"]:
            ms = {name: k[name + "_ms"] for name in ("register", "tma")}
            assert all(v > 0 for v in ms.values())
            tuned = p["candidate"] in (2, 3)
            assert k["kernel"] == (min(ms, key=ms.get) if tuned else "register")
            if k["grid"] == [8, 8, 64]:
                assert k["plane_ms"] > 0 and k["onchip_ms"] > 0
                assert k["onchip"] == (tuned and k["onchip_ms"] < min(ms.values()) + k["plane_ms"])
            else:
                assert not k["onchip"]


def test_fused_plan_is_one_launch_per_step(monkeypatch, ground_states):
    monkeypatch.setenv("BEC_STEP_PLAN", "2")
    eng, groups = _three_classes(ground_states)
    p = eng.step_plan
    assert p["chosen"] == "forced" and p["fused_classes"] == 3
    eng.evolve(64)                                 # steady steps: captured graph replays
    assert eng.step_graphs == 2
    assert eng.last_launch_count == 64 * p["launches_per_step"] + 1   # + the step index write
    assert p["launches_per_step"] <= 2
    ms, cells = eng.profile_fused_step(3)
    assert ms > 0 and cells == sum(q.ne * q.nvx * q.nvy * q.nvz for q in groups)


def test_dependency_wait_that_runs_out_is_reported(monkeypatch, ground_states):
    monkeypatch.setenv("BEC_STEP_PLAN", "2")
    monkeypatch.setenv("BEC_STEP_WAIT_LIMIT_MS", "20")
    monkeypatch.setenv("BEC_STEP_INJECT_STALL", "1")
    eng = Engine([GROUPS[0]], path=BEC_PATH_FP32_BATCHED)
    eng.init_group(0, ground_states[0])
    with pytest.raises(BecError) as ei:
        eng.start_evolution()
    assert ei.value.status == BEC_ERR_CUDA and "wait" in str(ei.value)
    eng.close()
    monkeypatch.delenv("BEC_STEP_INJECT_STALL")
    monkeypatch.delenv("BEC_STEP_WAIT_LIMIT_MS")
    got = _run(monkeypatch, "2", ground_states[:1], groups=[GROUPS[0]])
    ref = _run(monkeypatch, "unfused", ground_states[:1], groups=[GROUPS[0]])
    np.testing.assert_array_equal(got["mom"], ref["mom"])


def test_tma_tile_wait_that_runs_out_is_reported(monkeypatch, ground_states):
    monkeypatch.setenv("BEC_STEP_PLAN", "unfused-tma")
    monkeypatch.setenv("BEC_STEP_WAIT_LIMIT_MS", "20")
    monkeypatch.setenv("BEC_PENCIL_INJECT_STALL", "1")
    eng = Engine([GROUPS[2]], path=BEC_PATH_FP32_BATCHED)
    eng.init_group(0, ground_states[2])
    with pytest.raises(BecError) as ei:
        eng.start_evolution()
    assert ei.value.status == BEC_ERR_CUDA and "wait" in str(ei.value)
    eng.close()
    monkeypatch.delenv("BEC_PENCIL_INJECT_STALL")
    monkeypatch.delenv("BEC_STEP_WAIT_LIMIT_MS")
    got = _run(monkeypatch, "unfused-tma", ground_states[2:3], groups=[GROUPS[2]])
    ref = _run(monkeypatch, "unfused", ground_states[2:3], groups=[GROUPS[2]])
    np.testing.assert_array_equal(got["mom"], ref["mom"])
    for a, b in zip(got["states"], ref["states"]):
        np.testing.assert_array_equal(a, b)
