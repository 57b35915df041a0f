"""Benchmark: Wigner trajectory-steps per second of the batched FP32 path.

Workload (the batched uneven-ensemble configuration): 1024 trajectories per
GPU in one context, grids drawn uniformly from 8x8x64, 16x16x128 and
32x32x256, N ~ U[5000, 70000], trap frequencies jittered +-10 %, Rb-87
two-body and three-body losses with Wigner loss noise, dt = 40 us. A step is
one split step of every trajectory. Initial states are Thomas-Fermi profiles
plus Philox vacuum noise (the cost of a step does not depend on the state).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One JSON line on rank 0. Under torchrun the ranks share one global batch of
1024 trajectories per GPU (weak scaling), sharded by cells; the timed region
is the max over ranks and the per-sample moments are all-reduced once.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# ncu: DRAM bytes (read + write) per cell of one launch of a pass kernel, from a capture of 64 x 32x32x256
# trajectories (268 MB of state, larger than L2; dram__bytes_read.sum + dram__bytes_write.sum over the launch's
# cells); traffic scales with the cells a launch processes (algorithmic: 32 B per cell).
NCU_TRAFFIC_PER_CELL = {"plane_32x32x256": 28.44, "pencil_32x32x256": 28.47}

# ncu: thread-instructions per cell of one launch (smsp__inst_executed.sum x 32 / cells), from the same
# capture. With the launch time they give the kernel's instruction issue rate, whose ceiling is one
# warp-instruction per scheduler per clock: SMs x 4 x 32 thread-instructions per clock.
NCU_INSTR_PER_CELL = {"plane_32x32x256": 354.9, "pencil_32x32x256": 131.8}

N_TRAJ = 1024
# stopping rules of the ground-state leg: |d mu|/mu between checks below 1e-7 stops every held-out set
# within 1e-6 of its converged mu (measured); 1e-6 is the reference-style test on the change alone
GS_TOL, GS_REF_TOL = 1e-7, 1e-6
GS_TRAIN_STEPS = 120000    # Adam steps: 10.6x on one box against 9.3x at 60000 (35 s of training)
WORKLOAD = "uneven-ensembles-1024"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="bec", choices=["bec", "reference"])
    ap.add_argument("--n-traj", type=int, default=N_TRAJ)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target length of the CPU baseline sample")
    ap.add_argument("--no-extras", action="store_true", help="skip the plain-path and CPU baseline legs")
    ap.add_argument("--no-gs", action="store_true", help="skip the warm-start ground-state leg")
    ap.add_argument("--gs-train", type=int, default=4096, help="training ground states of the warm-start leg")
    ap.add_argument("--gs-eval", type=int, default=256, help="held-out parameter sets of the warm-start leg")
    ap.add_argument("--grids", default=None,
                    help="restrict the grid mix, e.g. 32x32x256 or 8x8x64,16x16x128 (profiling captures)")
    return ap.parse_args()


def grid_mix(args):
    from bec_b200.configs import UNEVEN_GRIDS
    if not args.grids:
        return UNEVEN_GRIDS
    return tuple(tuple(int(v) for v in g.split("x")) for g in args.grids.split(","))


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def thomas_fermi(d):
    import numpy as np
    x = -d.xmax + d.dx * np.arange(d.nvx)
    y = (-d.ymax + d.dy * np.arange(d.nvy)) if d.nvy > 1 else np.zeros(1)
    z = -d.zmax + d.dz * np.arange(d.nvz)
    V = (x[None, None, :] ** 2 + y[None, :, None] ** 2 + z[:, None, None] ** 2 / d.lambda_ ** 2) / 2
    return np.sqrt(np.maximum(d.mu - V, 0.0) / d.g11).reshape(-1).astype(np.complex128)


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.f:
            return None
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for k, n in enumerate(names):
                    if r[5 + k].strip().lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        j = json.load(open(p))
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def mix_sample(groups, n):
    """n trajectories of groups (one trajectory per group) with the batch's share of every grid class, so that a
    sample's traj-steps/s compare with the whole batch's (the first ones of each class, in batch order)."""
    by = {}
    for p in groups:
        by.setdefault((p.nvx, p.nvy, p.nvz), []).append(p)
    n = min(n, len(groups))
    share = {k: n * len(v) / len(groups) for k, v in by.items()}
    take = {k: int(x) for k, x in share.items()}
    for k in sorted(share, key=lambda q: take[q] - share[q])[:n - sum(take.values())]:
        take[k] += 1                                   # largest remainders first
    out, used = [], {k: 0 for k in take}
    for p in groups:
        k = (p.nvx, p.nvy, p.nvz)
        if used[k] < take[k]:
            out.append(p)
            used[k] += 1
    return out


def mean_cells(groups):
    return sum(p.nvx * p.nvy * p.nvz * p.ne for p in groups) / max(1, sum(p.ne for p in groups))


def host_cpu():
    """The host's CPU model, its logical CPU count and how many of those this process may run on."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count() or 1
    return {"cpu_model": model, "nproc": os.cpu_count(), "usable_cpus": usable}


class OracleSample:
    """A bounded sample of the workload on the CPU oracle (FP64 restatement of the
    reference's split step), one trajectory per thread on all host cores the process may use;
    the sample has the workload's grid-class mix."""

    def __init__(self, groups):
        from concurrent.futures import ThreadPoolExecutor
        from oracle import oracle as O
        self.cores = host_cpu()["usable_cpus"]
        self.sample = mix_sample(groups, max(3, 2 * self.cores))
        self.ens = []
        for p in self.sample:
            e = O.OracleEnsemble(p)
            e.init(thomas_fermi(O.derive(p)))
            self.ens.append(e)
        self.pool = ThreadPoolExecutor(max_workers=self.cores)

    def step(self):
        """One split step of every sampled trajectory; returns the wall time."""
        t0 = time.perf_counter()
        list(self.pool.map(lambda e: e.evolve(1, 1), self.ens))
        return time.perf_counter() - t0

    def step_serial(self):
        """The same step with every trajectory on the calling thread, one after another; returns the wall time."""
        t0 = time.perf_counter()
        for e in self.ens:
            e.evolve(1, 1)
        return time.perf_counter() - t0

    def describe(self, steps, seconds):
        grids = {}
        for p in self.sample:
            k = f"{p.nvx}x{p.nvy}x{p.nvz}"
            grids[k] = grids.get(k, 0) + 1
        return f"{len(self.sample)} trajectories of the workload mix {grids}, {steps} steps, {seconds:.1f} s"

    def close(self):
        self.pool.shutdown()


def cpu_baseline(groups, seconds):
    """Oracle throughput on the sample for about `seconds` on all usable cores, then for about half as
    long on one thread: (traj-steps/s, cores, sample, single-thread record)."""
    s = OracleSample(groups)
    s.step()
    reps = max(1, int(seconds / max(s.step(), 1e-3)))
    el = sum(s.step() for _ in range(reps))
    v = len(s.sample) * reps / el
    first = s.step_serial()
    reps1 = max(1, int(0.5 * seconds / max(first, 1e-3)))
    el1 = sum(s.step_serial() for _ in range(reps1))
    v1 = len(s.sample) * reps1 / el1
    s.close()
    single = {"value": v1, "unit": "traj-steps/s", "threads": 1,
              "sample": f"the same {len(s.sample)} trajectories one after another on one thread, {reps1} steps, "
                        f"{el1:.1f} s", "speedup_all_cores": v / v1, **host_cpu()}
    return v, s.cores, s.describe(reps, el), single


def run_reference(args, ws, rank):
    from bec_b200.configs import uneven_batch
    if rank != 0:
        return
    groups = uneven_batch(n_traj=args.n_traj, seed=2, grids=grid_mix(args))
    s = OracleSample(groups)
    for _ in range(args.warmup):
        s.step()
    # each bench step is one oracle step of the sample, capped so the run stays within minutes
    steps = min(args.steps, max(3, int(args.cpu_seconds * 6 / max(s.step(), 1e-3))))
    el = sum(s.step() for _ in range(steps))
    v = len(s.sample) * steps / el
    cores, sample = s.cores, s.describe(steps, el)
    s.close()
    line = {
        "impl": "reference", "metric": "wigner_traj_steps_per_s", "value": v, "unit": "traj-steps/s",
        "n_gpus": ws, "steps": steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD if not args.grids else f"{args.n_traj}x{args.grids}", "n_traj": args.n_traj,
                   "grids": args.grids or "8x8x64/16x16x128/32x32x256 uniform",
                   "step": "one split step of every trajectory of a bounded sample of the workload",
                   "implementation": "CPU FP64 restatement of the reference's split step (oracle port)"},
        "cpu_baseline": {"value": v, "unit": "traj-steps/s", "cores": cores, "kind": "port", "sample": sample,
                         **host_cpu()},
        "e2e": {"value": v, "unit": "traj-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def gs_warmstart_leg(n_train, n_eval, tol, ref_tol):
    """The ground-state half of the metric on the warm-start workload (32x32x256, N ~ U[5000, 100000],
    trap frequencies +-10 %, scattering lengths +-2 %): n_train ground states by the batched FP32 loop,
    the basis and the network trained on them on the device, then n_eval held-out sets from
    Thomas-Fermi (cold) and from the network's prediction (warm) under the same stopping rule; each
    result's mu is compared with the same set converged far beyond the rule (mu*)."""
    import numpy as np
    from bec_b200 import warmstart as W
    t0 = time.time()
    tr = W.sample_params(n_train, 3)
    ev = W.sample_params(n_eval, 4)
    # training ground states converged at the same accurate rule as the evaluation: the network learns
    # coefficients good to ~1e-3, not the ~2e-3 of states stopped at |d mu|/mu < 1e-6
    kw = dict(tol=tol, check_every=20, max_steps=40000)
    n_pod = min(512, n_train)
    first = W.ground_states(tr[:n_pod], want_profiles=True, **kw)
    basis, _ = W.pod_basis(first["profiles"])
    c_tr = W.project(basis, first["profiles"])
    gen_s = first["seconds"]
    if n_train > n_pod:
        rest = W.ground_states(tr[n_pod:], basis=basis, **kw)
        c_tr = np.concatenate([c_tr, rest["coef"]])
        gen_s += rest["seconds"]
    t_train = time.time()
    ws, hist = W.train(tr, c_tr, steps=GS_TRAIN_STEPS)
    t_train = time.time() - t_train
    ref = W.ground_states(ev, basis=basis, tol=1e-10, res_tol=1e-9, check_every=20, max_steps=40000)
    mu_star = ref["mu"]
    pred_t = time.time()
    pred = ws.predict(ev)
    t_inf = time.time() - pred_t

    def leg(rule_tol):
        cold = W.ground_states(ev, basis=basis, tol=rule_tol, check_every=20, max_steps=40000)
        warm = W.ground_states(ev, coef_in=pred, basis=basis, tol=rule_tol, check_every=20, max_steps=40000)
        return {
            "rule": f"|d mu|/mu < {rule_tol:g} between checks and fixed-point residual < {10 * rule_tol:g}, "
                    "checked every 20 steps (BEC_GS_MU_RESIDUAL)",
            "cold_s": cold["seconds"], "warm_s": warm["seconds"] + t_inf,
            "speedup_s": cold["seconds"] / max(warm["seconds"] + t_inf, 1e-12),
            "cold_steps_mean": float(cold["steps"].mean()), "warm_steps_mean": float(warm["steps"].mean()),
            "speedup_steps": float(cold["steps"].mean() / max(warm["steps"].mean(), 1.0)),
            "cold_mu_err_max": float(np.max(np.abs(cold["mu"] - mu_star) / mu_star)),
            "warm_mu_err_max": float(np.max(np.abs(warm["mu"] - mu_star) / mu_star)),
            "converged": [float(cold["converged"].mean()), float(warm["converged"].mean())],
        }

    accurate = leg(tol)
    # the basis's own limit: warm starts from the held-out sets' converged coefficients (a diagnostic beside the
    # network's warm start, not a product path)
    bound = W.ground_states(ev, coef_in=ref["coef"], basis=basis, tol=tol, check_every=20, max_steps=40000)
    return {
        "workload": f"32x32x256 warm-start ground states, {n_train} training / {n_eval} held-out parameter sets",
        "unit": "s (device time of the held-out batch; warm includes the network's inference)",
        **accurate,
        "reference_rule": leg(ref_tol),
        "projection_bound": {"note": "warm starts from the held-out sets' own converged coefficients, accurate rule",
                             "warm_s": bound["seconds"], "warm_steps_mean": float(bound["steps"].mean()),
                             "speedup_s": accurate["cold_s"] / max(bound["seconds"], 1e-12)},
        "mu_star": f"each held-out set run on to |d mu|/mu < 1e-10 and residual < 1e-9 or 40000 steps "
                   f"({float(ref['steps'].mean()):.0f} steps mean); the FP32 fixed point lies 3e-7 to 4e-7 from "
                   "the FP64 one",
        "inference_s": t_inf,
        "training": {"ground_states_device_s": gen_s, "rule": f"|d mu|/mu < {tol:g}, residual < {10 * tol:g}",
                     "adam_steps": GS_TRAIN_STEPS, "train_s": t_train, "loss_last": float(hist[-10:].mean())},
        "wall_s": time.time() - t0,
    }


def physical_gpu_index(dev):
    """nvidia-smi index of CUDA device `dev` (nvidia-smi ignores CUDA_VISIBLE_DEVICES)."""
    entries = [e.strip() for e in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if e.strip()]
    if dev < len(entries) and entries[dev].isdigit():
        return int(entries[dev])
    return dev


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        if ws > 1:
            import torch.distributed as dist
            dist.init_process_group("gloo")
        run_reference(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import numpy as np
    import torch
    from bec_b200 import distributed as D
    from bec_b200.configs import uneven_batch
    from bec_b200.engine import BEC_PATH_FP32_BATCHED, BEC_PATH_FP64_PLAIN, Engine

    # one GPU per rank: LOCAL_RANK among the visible devices (every GPU stays visible, so NCCL sees its
    # peers), or device 0 when the launcher already gives each rank a single visible GPU
    dev = local if local < torch.cuda.device_count() else 0
    torch.cuda.set_device(dev)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    # one global uneven ensemble of n_traj trajectories per GPU (weak scaling), sharded over the ranks by
    # cells (longest first); each rank's context holds its shard, and the only exchange is the FP64
    # all-reduce of the per-sample moments of every ensemble
    all_groups = uneven_batch(n_traj=args.n_traj * ws, seed=2, grids=grid_mix(args))
    mine = D.shard(all_groups, rank, ws)
    groups = [all_groups[i] for i in mine]
    eng = Engine(groups, path=BEC_PATH_FP32_BATCHED)
    # pinned host ground states (Thomas-Fermi), reused by the e2e leg
    host_gs = []
    for g, d in enumerate(eng.derived):
        tf = thomas_fermi(d)
        pin = torch.empty(2 * d.cells, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128)
        pin[:] = tf
        host_gs.append(pin)
    for g in range(eng.n_groups):
        eng.init_group(g, host_gs[g])
    eng.start_evolution()
    cells = np.array([d.cells for d in eng.derived], dtype=np.float64)
    total_cells = float(cells.sum())

    # warm-up, then K device-timed steps
    eng.evolve(args.warmup)     # the first steps also run the schedule autotuner
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    with ClockSampler(physical_gpu_index(dev)) as clk:
        eng.evolve(args.steps)
        torch.cuda.synchronize()
    ms = eng.last_device_ms
    launches = eng.last_launch_count
    if ws > 1:
        dist.barrier()
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    n_traj_total = len(all_groups)
    value = n_traj_total * args.steps / (ms * 1e-3)

    # device time of the dominant kernel: the fused step kernel (one launch per step covering every grid
    # class, CUDA events on the engine's stream), and the per-pass kernels of the launch-per-pass schedule
    plan = eng.step_plan
    peak, peak_kind = peaks()
    prof = eng.profile_steps(3)
    kernels = []
    for c in prof:
        nx, ny, nz = c["dims"]
        bytes_launch = 32.0 * nx * ny * nz * c["traj"]      # read + write of both complex64 components
        for kind, t in (("pencil", c["z_ms"]), ("plane", c["plane_ms"])):
            kernels.append(dict(kernel=f"{kind}_{nx}x{ny}x{nz}", ms=t, bytes=bytes_launch,
                                cells=nx * ny * nz * c["traj"]))
    per_pass = {k["kernel"]: {"ms": k["ms"], "frac": k["bytes"] / (k["ms"] * 1e-3) / 1e9 / peak} for k in kernels}
    if plan.get("fused_classes", 0) > 0:
        # the fused step kernel: one launch per step covering every register-path class
        fused_ms, fused_cells = eng.profile_fused_step(5)
        dom = dict(kernel="k_step", ms=fused_ms, bytes=32.0 * fused_cells, cells=fused_cells,
                   label="k_step (fused split step, every grid class, one launch)",
                   note="32 B per cell and step (both complex64 components read and written once); the kernel "
                        "does both passes of the step")
    else:
        # per-pass launches (the autotuner's choice): the longest of them
        dom = max(kernels, key=lambda k: k["ms"])
        dom = dict(dom, label=dom["kernel"], note="32 B per cell of the class per launch (one pass of the step)")
    achieved = dom["bytes"] / (dom["ms"] * 1e-3) / 1e9
    traffic = NCU_TRAFFIC_PER_CELL[dom["kernel"]] * dom["cells"] if dom["kernel"] in NCU_TRAFFIC_PER_CELL else None
    roofline = {"bound": "hbm", "kernel": dom["label"], "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic, "algorithmic_bytes": dom["bytes"],
                "ms_per_launch": dom["ms"], "note": dom["note"]}
    step_gbs = 32.0 * total_cells * args.steps / (ms * 1e-3) / 1e9 * (ws if ws > 1 else 1)
    step_roof = {"achieved": step_gbs / ws if ws > 1 else step_gbs, "peak": peak, "unit": "GB/s",
                 "frac": (step_gbs / ws if ws > 1 else step_gbs) / peak,
                 "note": "32 B/cell/step algorithmic bytes of the whole step, all kernels"}

    # e2e through the C ABI: host ground states (pinned, real FP32: the ground states are real, and the FP32
    # path rounds them to FP32 on the device either way) -> one batched init of every ensemble -> pi/2 ->
    # K steps -> moments to host; one pinned buffer, the groups' ground states back to back in group order
    # (bec_init_groups then copies them in one transfer)
    pin = torch.empty(sum(a.size for a in host_gs), dtype=torch.float32, pin_memory=True).numpy()
    host_gs64, o = [], 0
    for a in host_gs:
        pin[o:o + a.size] = a.real
        host_gs64.append(pin[o:o + a.size])
        o += a.size
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    t0 = time.perf_counter()
    eng.init_groups(range(eng.n_groups), host_gs64)
    eng.start_evolution()
    every = max(1, args.steps // 4)
    mom = eng.run(args.steps, sample_every=every)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if ws > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = 4.0 * total_cells / args.steps
    d2h = 40.0 * mom.shape[0] * mom.shape[1] / args.steps
    e2e = {"value": n_traj_total * args.steps / e2e_s, "unit": "traj-steps/s",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "note": "batched init from pinned real FP32 host ground states + pi/2 + K steps + moments to host, per call"}

    # ensemble observables of the global batch: one small FP64 all-reduce of the per-sample moments
    mom_all = D.allreduce_moments(mom, mine, len(all_groups), device="cuda")
    assert mom_all.shape[1] == len(all_groups)

    extras = {}
    cpu = None
    if rank == 0 and ws == 1 and not args.no_extras:
        # plain per-trajectory FP64 path on a sample with the batch's grid mix
        sample = mix_sample(groups, 24)
        plain = Engine(sample, path=BEC_PATH_FP64_PLAIN)
        for g, d in enumerate(plain.derived):
            plain.init_group(g, thomas_fermi(d))
        plain.start_evolution()
        plain.evolve(2)
        plain_steps = 20
        plain.evolve(plain_steps)
        pv = len(sample) * plain_steps / (plain.last_device_ms * 1e-3)
        # the batched path on the same sample, for the like-for-like ratio
        bs = Engine(sample, path=BEC_PATH_FP32_BATCHED)
        for g, d in enumerate(bs.derived):
            bs.init_group(g, thomas_fermi(d))
        bs.start_evolution()
        bs.evolve(3)
        bs.evolve(10)
        bv = len(sample) * 10 / (bs.last_device_ms * 1e-3)
        mix = {}
        for p in sample:
            mix[f"{p.nvx}x{p.nvy}x{p.nvz}"] = mix.get(f"{p.nvx}x{p.nvy}x{p.nvz}", 0) + 1
        extras["plain_fp64"] = {"value": pv, "unit": "traj-steps/s",
                                "sample": f"{len(sample)} trajectories of the workload mix {mix}, {plain_steps} steps",
                                "batched_fp32_same_sample": bv, "ratio_same_sample": bv / pv,
                                "ratio_full_batch": value / pv}
        plain.close()
        bs.close()
        v, cores, s, single = cpu_baseline(groups, args.cpu_seconds)
        cpu = {"value": v, "unit": "traj-steps/s", "cores": cores, "kind": "port", "sample": s,
               "cell_steps_per_s": v * mean_cells(mix_sample(groups, max(3, 2 * cores))),
               "single_thread": single}
    if rank == 0 and ws == 1 and not args.no_extras and not args.no_gs:
        extras["gs_warmstart"] = gs_warmstart_leg(args.gs_train, args.gs_eval, GS_TOL, GS_REF_TOL)

    clocks = clk.summary()
    issue_roof = None
    if dom["kernel"] in NCU_INSTR_PER_CELL:
        instr = NCU_INSTR_PER_CELL[dom["kernel"]] * dom["cells"]
        mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz")
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        if mhz:
            ach = instr / (dom["ms"] * 1e-3)
            pk = sms * 4 * 32 * mhz * 1e6
            issue_roof = {"kernel": dom["kernel"], "thread_instructions_per_cell": NCU_INSTR_PER_CELL[dom["kernel"]],
                          "achieved": ach, "peak": pk, "unit": "thread-instr/s", "frac": ach / pk,
                          "note": "instruction issue, the bound of this kernel: one warp-instruction per scheduler "
                                  "per clock at the sampled SM clock; instructions per cell from ncu"}
    # the transforms' FLOPs (5 n log2 n per complex transform of n points; two components, one inverse and
    # one forward 3D transform per step) against the FP32 FMA pipes: the compute bound beside the HBM bound
    flop_roof = None
    mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz")
    if mhz:
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        flops = float(np.sum(20.0 * cells * np.log2(cells)))
        step_s = ms / args.steps * 1e-3
        pk = sms * 128 * 2 * mhz * 1e6
        t_flop, t_hbm = flops / pk, 32.0 * total_cells / (peak * 1e9)
        flop_roof = {"achieved": flops / step_s / 1e12, "peak": pk / 1e12, "unit": "TFLOP/s",
                     "frac": flops / step_s / pk, "flop_per_byte": flops / (32.0 * total_cells),
                     "flop_time_ms": t_flop * 1e3, "hbm_time_ms": t_hbm * 1e3,
                     "ceiling_ms": max(t_flop, t_hbm) * 1e3, "ms_per_step": ms / args.steps,
                     "note": "whole step, this GPU's trajectories: transform FLOPs only (the cell step, Philox and "
                             "Box-Muller add more); peak = the FP32 FMA pipes' nominal 2 flop per lane per clock at "
                             "the sampled SM clock (the measured peaks hold no FP32 figure); ceiling = the slower of "
                             "the FLOP and the HBM time"}
    if rank == 0:
        line = {
            "metric": "wigner_traj_steps_per_s", "value": value, "unit": "traj-steps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "cell_steps_per_s": value * mean_cells(all_groups),
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD if not args.grids else f"{args.n_traj}x{args.grids}",
                       "n_traj_per_gpu": args.n_traj,
                       "grids": args.grids or "8x8x64/16x16x128/32x32x256 uniform", "N": "U[5000,70000]",
                       "trap_jitter": "+-10%", "dt_s": 4e-5, "noise": "Philox vacuum + loss noise",
                       "l2": f"state {16 * total_cells / 1e9:.2f} GB per GPU, larger than L2",
                       "parallelism": f"dp{ws} (trajectory sharding)", "path": "fp32-batched"},
            "roofline": roofline, "issue_roofline": issue_roof, "step_roofline": step_roof,
            "flop_roofline": flop_roof,
            "step_plan": plan, "per_pass_kernels": per_pass, "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches, "clocks": clocks, **extras,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
