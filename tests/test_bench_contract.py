"""The benchmark's output contract: one JSON line with the keys a driver reads.

The reference arm (the FP64 CPU restatement of the reference's split step) runs here on the CPU on
a small sample. The GPU arm runs a small workload on a B200. Both must print exactly one JSON line
with the metric, its unit and the objects the bench line promises.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bench_line(args, env=None):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                       cwd=ROOT, env=env, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def test_reference_arm_line():
    d = bench_line(["--impl", "reference", "--steps", "1", "--warmup", "0", "--n-traj", "8", "--cpu-seconds", "1"])
    assert d["impl"] == "reference"
    assert d["metric"] == "wigner_traj_steps_per_s" and d["unit"] == "traj-steps/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert cb["nproc"] >= cb["usable_cpus"] == cb["cores"] >= 1 and "cpu_model" in cb
    assert d["e2e"] == {"value": d["value"], "unit": "traj-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_under_torchrun_prints_one_line():
    """Launched like the multi-GPU bench (torchrun, two ranks, gloo here), the reference arm runs on rank 0
    alone: exactly one JSON line, every rank exits 0."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
                        "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--n-traj", "8",
                        "--cpu-seconds", "1"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0


def test_baseline_samples_keep_the_batch_mix():
    """The CPU and plain-FP64 baseline samples hold every grid class in the batch's proportion (largest
    remainders), so their traj-steps/s compare with the batch's."""
    sys.path.insert(0, ROOT)
    import bench
    from bec_b200.configs import uneven_batch
    groups = uneven_batch(n_traj=1024, seed=2)
    counts = {}
    for p in groups:
        counts[(p.nvx, p.nvy, p.nvz)] = counts.get((p.nvx, p.nvy, p.nvz), 0) + 1
    for n in (3, 24, 32, 100):
        s = bench.mix_sample(groups, n)
        assert len(s) == n and len({id(p) for p in s}) == n
        got = {}
        for p in s:
            got[(p.nvx, p.nvy, p.nvz)] = got.get((p.nvx, p.nvy, p.nvz), 0) + 1
        for k, c in counts.items():
            assert abs(got.get(k, 0) - n * c / len(groups)) < 1.0
    assert bench.mix_sample(groups[:5], 32) == groups[:5]


def test_cpu_baseline_times_all_cores_and_one_thread():
    """The CPU baseline times the oracle on every usable core and, on the same sample, on one thread, and
    names the host's CPU."""
    sys.path.insert(0, ROOT)
    import bench
    from bec_b200.configs import uneven_batch
    groups = uneven_batch(n_traj=6, seed=2, grids=[(8, 8, 64)])
    v, cores, sample, single = bench.cpu_baseline(groups, 0.2)
    assert v > 0 and cores == bench.host_cpu()["usable_cpus"] and "8x8x64" in sample
    assert single["threads"] == 1 and single["value"] > 0 and single["unit"] == "traj-steps/s"
    assert single["speedup_all_cores"] == v / single["value"]
    assert single["nproc"] >= single["usable_cpus"] >= 1 and "one thread" in single["sample"]


def test_rank_to_physical_gpu(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.delenv("CUDA_VISIBLE_DEVICES", raising=False)
    assert bench.physical_gpu_index(3) == 3
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "4,5,6,7")
    assert bench.physical_gpu_index(0) == 4 and bench.physical_gpu_index(3) == 7
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "GPU-abc")       # UUIDs: fall back to the CUDA index
    assert bench.physical_gpu_index(0) == 0


@pytest.mark.gpu
def test_gpu_arm_line():
    d = bench_line(["--steps", "5", "--warmup", "3", "--n-traj", "48", "--no-extras"])
    assert d["metric"] == "wigner_traj_steps_per_s" and d["value"] > 0 and d["steps"] == 5 and d["warmup"] == 3
    roof = d["roofline"]
    assert roof["bound"] == "hbm" and roof["peak"] > 0 and 0 < roof["frac"] == pytest.approx(roof["achieved"] / roof["peak"])
    e2e = d["e2e"]
    assert e2e["value"] > 0 and e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    assert d["gpu_launches"] > 0
    if d["clocks"] is not None:                 # None only where nvidia-smi gave no samples
        assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(d["clocks"])
        fr = d["flop_roofline"]
        assert fr["unit"] == "TFLOP/s" and 0 < fr["frac"] == pytest.approx(fr["achieved"] / fr["peak"])
        assert fr["ceiling_ms"] == max(fr["flop_time_ms"], fr["hbm_time_ms"]) <= fr["ms_per_step"]
