"""Benchmark: batch edge collision checking, edges/s (panda, 1000 envs).

One step = one batched check of the uneven workload (1000 environments with
U{8..64} primitives x 10000 edges of log-uniform length 0.05-2.0 rad, seeded
synthetic data) through the checker; a verdict for every (env, edge) pair.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--order plain|learned]

Multi-GPU (torchrun, one rank per GPU): every rank checks its own edge set
against the same environments (weak scaling, no data-path collective); time
is the max over ranks.  `--impl reference` times the reference algorithm on the
host cores (the CPU restatement in oracle/, all threads), or with
`--ref-path cuda` the reference's own CUDA kernel (oracle/_ref).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "batch-cc_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOAD = "uneven"
METRIC = "edges/sec (panda, 1000 envs) learned-ordered vs plain; verdict mismatches=0"
UNIT = "edges/s"
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


COUNTS_FILE = os.path.join("profiles", "check_kernel_counts.md")


def committed_counts(workload_name_):
    """Per-pair counts of the plain-order check kernel on a workload, from the
    committed ncu summary: warp instructions executed, FP32 FFMA / FADD / FMUL
    thread instructions and DRAM bytes, each divided by the pairs of the
    captured launch (None when the workload has no capture)."""
    import re
    path = os.path.join(ROOT, COUNTS_FILE)
    if not os.path.exists(path):
        return None
    m = re.search(r"^counts %s (.*)$" % re.escape(workload_name_), open(path).read(), re.M)
    if not m:
        return None
    f = m.group(1).split()
    return {f[i]: float(f[i + 1]) for i in range(0, len(f) - 1, 2)}


def metric_of(name, N):
    """The headline metric on the headline workload; the same quantity, named
    for its robot and size, on the others."""
    from bcc import workload
    if name == WORKLOAD:
        return METRIC
    return "edges/sec (%s, %d envs) learned-ordered vs plain; verdict mismatches=0" % (workload.robot_of(name), N)


def workload_name(name, N, E):
    """Human-readable workload description (robot, sizes, size laws)."""
    from bcc import workload
    w = workload.WORKLOADS[name]
    prims = "8 spheres, 8 cuboids, 4 cylinders" if w["prims"] == "fixed" else "U{%d..%d} primitives" % w["prims"]
    edges = "uniform in the joint limits" if w["edge_law"] == "uniform" else "log-uniform 0.05-2.0 rad"
    return "%s: %s, %d envs (%s) x %d edges (%s)" % (name, w["robot"], N, prims, E, edges)


def bench_config(name, N, E, world):
    """The workload description both arms print, key for key."""
    return {"workload": "%s, resolution 32" % workload_name(name, N, E), "envs": N, "edges_per_gpu": E,
            "resolution": 32, "l2": "256 MB buffer written between timed steps (untimed)",
            "parallelism": "dp%d" % world}


def parity_vs_reference(envs, edges, verdicts, robot, iters=3):
    """Checker leg, untimed and after the timed region: the reference's own CUDA
    kernel batch_cc_kernel<Robot> (src/batch_cc.cu:74-133, built unmodified from
    the reference sources into oracle/_ref) on the same inputs; every verdict of
    each order is compared with it and each mismatch adjudicated by the FP64
    signed penetration of the pair (oracle): within 1e-5 m of contact it is
    tolerated, beyond it counts as out of tolerance.  Also returns the reference
    kernel's throughput, CUDA-event timed (mean of `iters` launches).  (None,
    None) when the reference harness was not built."""
    from oracle import oracle as orc
    from oracle import ref
    if not ref.available():
        return None, None
    N, E = envs.num_envs, len(edges)
    ms, want = ref.time_kernel(envs, edges, iters=iters, robot=robot)
    par = {"pairs": int(want.size),
           "vs": "reference CUDA batch_cc_kernel<%s> (src/batch_cc.cu:74-133), built from the reference sources"
                 % robot.capitalize(),
           "tolerance": "mismatch tolerated when the FP64 penetration of the pair is within 1e-5 m of contact"}
    worst = 0
    for order, got in verdicts.items():
        n_mis, n_adj, bad = orc.adjudicate(envs, edges, got, want, robot=robot)
        par[order] = {"mismatches": int(n_mis), "mismatches_adjudicated": int(n_adj),
                      "mismatches_out_of_tolerance": int(len(bad))}
        worst = max(worst, int(len(bad)))
        par.setdefault("mismatches_adjudicated", 0)
        par["mismatches_adjudicated"] = max(par["mismatches_adjudicated"], int(n_adj))
    par["mismatches_out_of_tolerance"] = worst
    ref_cuda = {"value": N * E / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                "timing": "CUDA events around the reference kernel launch, mean of %d" % iters,
                "kernel": "batch_cc_kernel<%s>, <<<N*E, 32>>>" % robot.capitalize()}
    return par, ref_cuda


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--ref-path", default="cpu", choices=["cpu", "cuda"])
    p.add_argument("--order", default="learned", choices=["plain", "learned"],
                   help="order whose throughput is the headline value (both are timed)")
    p.add_argument("--train-samples", type=int, default=10_000_000)
    p.add_argument("--train-epochs", type=int, default=2)
    p.add_argument("--train-envs", type=int, default=4000)
    p.add_argument("--workload", default=WORKLOAD)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-parity", action="store_true", help="skip the full-size parity leg against the reference "
                                                             "CUDA kernel")
    p.add_argument("--flop-sample", type=int, default=20000)
    p.add_argument("--no-others", action="store_true", help="skip the Fetch, Baxter and stress workloads")
    p.add_argument("--profile-order", default=None, choices=["plain", "learned"],
                   help="profiling run: only `--warmup` + `--steps` eager checks in this order (launch config "
                        "--profile-launch, MLP at its seeded initialisation), no training, tuning or baselines")
    p.add_argument("--profile-launch", default="128,4,0",
                   help="edges per CTA, warps per CTA, persistent (0/1) and optionally the learned-order queue "
                        "threshold of a profiling run; the default is the configuration the autotuner picks for "
                        "the plain order of the uneven workload")
    p.add_argument("--envs", type=int, default=None, help="smaller case for profiling")
    p.add_argument("--edges", type=int, default=None, help="smaller case for profiling")
    return p.parse_args()


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        if args.impl == "ours":  # the reference arm runs on the host cores (gloo), no GPU needed
            torch.cuda.set_device(local)
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def rank_edges(workload_name_, num_edges, rank):
    """Each rank checks its own seeded edge set against the same environments
    (weak scaling: per-rank work fixed as ranks are added)."""
    from bcc import workload
    return workload.gen_edges(workload_name_, num_edges, seed=rank)


def max_over_ranks(dist, v, device):
    """The largest of every rank's value (identity without a process group)."""
    if not dist:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(envs, edges, robot="panda", target_s=12.0):
    """The CPU restatement of the reference algorithm (oracle, FP32, all host
    threads) on a bounded sample: all environments x the first edges."""
    from oracle import oracle as orc
    cores = os.cpu_count() or 1
    n_e = 100
    t0 = time.perf_counter()
    orc.check(envs, edges[:n_e], precision=32, nthreads=cores, robot=robot)
    dt = time.perf_counter() - t0
    n_e2 = int(min(len(edges), max(n_e, n_e * target_s / max(dt, 1e-3))))
    t0 = time.perf_counter()
    orc.check(envs, edges[:n_e2], precision=32, nthreads=cores, robot=robot)
    dt = time.perf_counter() - t0
    return {"value": n_e2 * envs.num_envs / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d envs x first %d edges of the workload (%.1f s), FP32 CPU restatement of the "
                      "reference algorithm (oracle/oracle.cpp), not VAMP" % (envs.num_envs, n_e2, dt)}


def algorithmic_flops(envs, edges, sample, robot="panda"):
    """Reference plain-order FLOPs per pair (oracle count), averaged over a seeded
    uniform sample of (edge, env) pairs, times all pairs."""
    from oracle import oracle as orc
    rng = np.random.default_rng(123)
    pairs = np.stack([rng.integers(0, len(edges), sample), rng.integers(0, envs.num_envs, sample)], 1)
    fl, _ = orc.pair_flops(envs, edges, pairs, robot=robot)
    return float(fl.mean()) * len(edges) * envs.num_envs, float(fl.std() / np.sqrt(sample) / fl.mean())


def run_reference(args, world, rank):
    from bcc import workload
    if rank != 0:
        return
    robot = workload.robot_of(args.workload)
    envs = workload.gen_envs(args.workload, args.envs, seed=0)
    edges = workload.gen_edges(args.workload, args.edges, seed=0)
    N, E = envs.num_envs, len(edges)
    cfg = bench_config(args.workload, N, E, world)
    if args.ref_path == "cuda":
        from oracle import ref
        if not ref.available():
            print(json.dumps({"impl": "reference", "unavailable": "reference harness oracle/_ref not built"}))
            return
        for _ in range(args.warmup):
            ref.time_kernel(envs, edges, iters=1, robot=robot)
        ms, _ = ref.time_kernel(envs, edges, iters=args.steps, robot=robot)
        val = N * E / (ms * 1e-3)
        t0 = time.perf_counter()
        ref.check(envs, edges, robot=robot)
        e2e_s = time.perf_counter() - t0
        line = {"metric": metric_of(args.workload, N), "value": val, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "config": cfg,
                "impl": "reference",
                "ref_path": "reference CUDA kernel batch_cc_kernel<%s> (oracle/_ref)" % robot.capitalize(),
                "e2e": {"value": N * E / e2e_s, "unit": UNIT,
                        "h2d_bytes_per_step": int(edges.nbytes), "d2h_bytes_per_step": N * E}}
        print(json.dumps(line))
        return
    from oracle import oracle as orc
    cores = os.cpu_count() or 1
    # Each step: a bounded sample (all envs x a fixed slice of edges), rotating slices.
    per_step = max(50, min(E, 400))
    for w in range(args.warmup):
        orc.check(envs, edges[:50], precision=32, nthreads=cores, robot=robot)
    t_tot = 0.0
    done = 0
    for s in range(args.steps):
        lo = (s * per_step) % E
        sl = edges[lo:lo + per_step]
        t0 = time.perf_counter()
        orc.check(envs, sl, precision=32, nthreads=cores, robot=robot)
        t_tot += time.perf_counter() - t0
        done += len(sl) * N
    val = done / t_tot
    ms = t_tot / args.steps * 1e3
    sample = "%d envs x %d edges per step, %d steps (%.1f s), FP32 CPU restatement of the reference " \
             "algorithm (oracle/oracle.cpp); the reference's VAMP CPU path is not vendored" % (
                 N, per_step, args.steps, t_tot)
    line = {"metric": metric_of(args.workload, N), "value": val, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def tune_edges(E, N):
    """Edges the autotuner times a configuration on: all of them up to 10 000,
    at most ~6e7 (env, edge) pairs per timed check, and at least 5000 edges
    when there are that many, so that the subset's sample table outgrows the
    126 MB L2 as the full one does (an L2-resident table favours the persistent
    kernel's environment-major order, which re-reads the table per environment
    once it does not fit: on the stress workload a tuning run on 2000 edges
    picked the persistent kernel, 729 ms per check, where an earlier run's grid
    kernel took 624 ms)."""
    return min(E, 10000, max(5000, 60_000_000 // max(N, 1)))


def plain_launches(robot):
    """Kernel launches of one plain-order check: Panda's row-major sample table
    has its self-collision check fused into the FK kernel."""
    return 5 if robot == "panda" else 6


TRAIN_QUEUE_MIN_ITEMS = 128  # the lowest queue threshold the tuner tries: its population holds every higher one's


def train_proposal(chk, args):
    """Train the collision-likelihood MLP (untimed) on the population the
    learned order acts on -- the segments of the pairs its probe queues --
    with checker labels, over environments and edges with seeds disjoint from
    the benchmark's."""
    from bcc import mlp, workload
    t0 = time.perf_counter()
    chk.upload(workload.gen_envs(args.workload, args.train_envs, seed=1000))
    chk.mlp_set_params(mlp.init_params(1000))
    train_edges = workload.gen_edges(args.workload, args.edges, seed=1000)
    losses, pos, rows = chk.mlp_train_queued(train_edges,
                                             num_samples=args.train_samples, queue_min_items=TRAIN_QUEUE_MIN_ITEMS,
                                             epochs=args.train_epochs, batch=16384, lr=2e-3, seed=1000,
                                             robot=workload.robot_of(args.workload))
    return {"train_rows": rows, "epochs": args.train_epochs, "epoch_loss": [float(v) for v in losses],
            "train_positive_fraction": pos, "train_seconds": time.perf_counter() - t0,
            "data": "segments (scored at their last sample) of the pairs the probe queues at threshold %d, "
                    "checker-labelled, %d %s environments x %d edges with seed 1000 (benchmark uses seed 0)" % (
                        TRAIN_QUEUE_MIN_ITEMS, args.train_envs, args.workload, len(train_edges))}


def proposal_ranking(chk, edges, queue_min_items, robot):
    """Ranking quality on the benchmark's own pairs that the first-sample probe
    leaves undecided with at least queue_min_items items to go (held out:
    trained on other seeds), for the trained network and for the same network
    untrained (its seeded initialisation), judged by the exact per-sample
    checks: AUC of the per-pair segment scores and the sample ranks walked to
    the first hit in the plain, learned and perfect orders
    (bcc_mlp_rank_metrics)."""
    from bcc import mlp
    trained = chk.mlp_get_params()
    out = {"population": "pairs left undecided by the probe of their first sample, >= %d items to go"
                         % queue_min_items,
           "queue_min_items": queue_min_items, "trained": chk.mlp_rank_metrics(edges, queue_min_items, robot=robot)}
    chk.mlp_set_params(mlp.init_params(1000))
    out["untrained"] = chk.mlp_rank_metrics(edges, queue_min_items, robot=robot)
    chk.mlp_set_params(trained)
    return out


def time_order(chk, d_edges, d_res, E, order, stream, steps, warmup, flush, dev, robot="panda", eager_reps=3):
    """Timed region: `steps` graph-captured (persistent-kernel) checks, L2 flushed
    between steps outside the timed events; then an untimed eager pass for the
    per-stage breakdown."""
    import torch

    def step(graph):
        chk.check_device(d_edges.data_ptr(), E, d_res.data_ptr(), order=order, stream=stream.cuda_stream, graph=graph,
                         robot=robot)

    for _ in range(warmup):
        step(True)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        flush.fill_(float(i))  # evict L2 between timed iterations (untimed)
        evs[i][0].record(stream)
        step(True)
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    total_ms = sum(x.elapsed_time(y) for x, y in evs)
    stage_tot, check_ms = {}, []
    reps = eager_reps
    for i in range(reps):
        flush.fill_(float(i))
        step(False)
        torch.cuda.synchronize()
        st = chk.stage_times()
        check_ms.append(st["check"])
        for k, v in st.items():
            stage_tot[k] = stage_tot.get(k, 0.0) + v
    return total_ms, check_ms, {k: v / max(reps, 1) for k, v in stage_tot.items()}


OTHER_WORKLOADS = ("multi_fetch", "multi_baxter", "stress")
# Parity subsample of the other workloads against the reference CUDA kernel:
# the first envs x first edges of the full inputs (all of them for Fetch and
# Baxter; 1000 x 10000 of the stress run's 10000 x 100000).
PARITY_SUBSAMPLE = {"multi_fetch": (500, 5000), "multi_baxter": (500, 5000), "stress": (1000, 10000)}


def measure_workload(chk, name, steps, warmup, flush, dev, parity, train_envs=2000, train_edges=5000):
    """One further workload at full size, compactly: the network trained on
    that workload's own queued population (seed 1000), launch configuration
    autotuned per order, both orders timed (graph replays, L2 flushed, CUDA
    events), verdicts of the orders compared, and parity against the
    reference CUDA kernel on a stated subsample (mismatches adjudicated)."""
    import torch
    from bcc import mlp, workload
    robot = workload.robot_of(name)
    stream = torch.cuda.current_stream()
    chk.upload(workload.gen_envs(name, train_envs, seed=1000))
    chk.mlp_set_params(mlp.init_params(1000))
    _, _, rows = chk.mlp_train_queued(workload.gen_edges(name, train_edges, seed=1000), num_samples=10_000_000,
                                      queue_min_items=TRAIN_QUEUE_MIN_ITEMS, epochs=2, batch=16384, lr=2e-3,
                                      seed=1000, robot=robot)
    envs = workload.gen_envs(name, seed=0)
    edges = workload.gen_edges(name, seed=0)
    N, E = envs.num_envs, len(edges)
    chk.upload(envs)
    d_edges = torch.from_numpy(edges).to(f"cuda:{dev}")
    d_res = torch.empty((E, N), dtype=torch.uint8, device=f"cuda:{dev}")
    d_res2 = torch.empty((E, N), dtype=torch.uint8, device=f"cuda:{dev}")
    n_tune = tune_edges(E, N)
    tuned = {o: chk.autotune(edges[:n_tune], order=o, robot=robot) for o in ("plain", "learned")}
    ms = {}
    for order, res in (("plain", d_res), ("learned", d_res2)):
        chk.set_launch_config(**tuned[order])
        total_ms, _, _ = time_order(chk, d_edges, res, E, order, stream, steps, warmup, flush, dev, robot,
                                    eager_reps=0)
        ms[order] = total_ms / steps
    learned_pairs = chk.last_learned_pairs()
    mismatch = int((d_res != d_res2).sum().item())
    out = {"workload": workload_name(name, N, E), "metric": metric_of(name, N), "unit": UNIT, "steps": steps,
           "warmup": warmup,
           "orders": {o: {"value": N * E / (ms[o] * 1e-3), "ms_per_step": ms[o], "launch": tuned[o]} for o in ms},
           "learned_over_plain": ms["plain"] / ms["learned"], "verdict_mismatches_learned_vs_plain": mismatch,
           "queued_pairs_per_step": learned_pairs, "train_rows": rows}
    if parity:
        nv, ne = PARITY_SUBSAMPLE[name]
        sub_envs = envs.subset(np.arange(min(nv, N)))
        verdicts = {"plain": d_res[:ne, :nv].cpu().numpy(), "learned": d_res2[:ne, :nv].cpu().numpy()}
        par, ref_cuda = parity_vs_reference(sub_envs, edges[:ne], verdicts, robot, iters=1)
        if par is not None:
            par["subsample"] = "first %d envs x first %d edges" % (sub_envs.num_envs, min(ne, E))
            out["parity"] = par
            out["reference_cuda"] = ref_cuda
    del d_res, d_res2, d_edges
    torch.cuda.empty_cache()
    return out


def mlp_roofline(chk, dev, rows=1 << 22, reps=5):
    """tcgen05 MLP forward kernel alone: 2 * rows * (48*128 + 2*128*128 + 128) FLOP per launch."""
    import torch
    x = torch.randint(-2000, 2000, (rows, 48), dtype=torch.int16, device=f"cuda:{dev}")
    x[:, 39:] = 0
    out = torch.empty(rows, dtype=torch.float32, device=f"cuda:{dev}")
    s = torch.cuda.current_stream()
    chk.mlp_forward_device(x.data_ptr(), rows, out.data_ptr(), stream=s.cuda_stream)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(reps):
        chk.mlp_forward_device(x.data_ptr(), rows, out.data_ptr(), stream=s.cuda_stream)
    b.record(s)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    flops = 2.0 * rows * (48 * 128 + 2 * 128 * 128 + 128)
    return ms, flops / (ms * 1e-3) / 1e12


def run_profile(args, local):
    """The check alone, for ncu: `warmup` + `steps` eager checks of the workload."""
    import torch
    from bcc import mlp, workload
    from bcc.lib import Checker

    torch.cuda.set_device(local)
    robot = workload.robot_of(args.workload)
    chk = Checker(local)
    envs = workload.gen_envs(args.workload, args.envs, seed=0)
    edges = workload.gen_edges(args.workload, args.edges, seed=0)
    chk.upload(envs)
    if args.profile_order == "learned":
        chk.mlp_set_params(mlp.init_params(1000))
    launch = [int(v) for v in args.profile_launch.split(",")]
    tile, warps, persistent = launch[:3]
    chk.set_launch_config(edges_per_cta=tile, warps=warps, persistent=persistent)
    if len(launch) > 3:
        chk.set_launch_config(queue_min_items=launch[3])
    if len(launch) > 4:
        chk.set_launch_config(finish_split=launch[4])
    for _ in range(args.warmup + args.steps):
        chk.check(edges, order=args.profile_order, robot=robot)
    torch.cuda.synchronize()
    chk.close()
    print(json.dumps({"profile": args.profile_order, "workload": workload_name(args.workload, envs.num_envs,
                                                                               len(edges)),
                      "checks": args.warmup + args.steps, "launch": args.profile_launch}))


def run_ours(args, world, rank, local, dist):
    import torch
    from bcc import workload
    from bcc.lib import Checker, measure_fp32_peak

    dev = local
    torch.cuda.set_device(dev)
    chk = Checker(dev)
    robot = workload.robot_of(args.workload)
    proposal = train_proposal(chk, args)
    envs = workload.gen_envs(args.workload, args.envs, seed=0)
    edges = rank_edges(args.workload, args.edges, rank)
    N, E = envs.num_envs, len(edges)
    chk.upload(envs)
    chk.set_profiling(True)
    stream = torch.cuda.current_stream()
    d_edges = torch.from_numpy(edges).to(f"cuda:{dev}")
    d_res = torch.empty((E, N), dtype=torch.uint8, device=f"cuda:{dev}")
    d_res2 = torch.empty((E, N), dtype=torch.uint8, device=f"cuda:{dev}")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{dev}")

    # Autotuned launch configuration per order (untimed), on the first edges.
    n_tune = tune_edges(E, N)
    tuned = {o: chk.autotune(edges[:n_tune], order=o, robot=robot) for o in ("plain", "learned")}
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    results = {}
    # Timed region: both orders, then the learned pipeline once more with the
    # network at its seeded initialisation (what the training itself adds),
    # each under the same clocks, launch and L2 flushes.
    from bcc import mlp as _mlp
    trained_params = chk.mlp_get_params()
    with ClockSampler(dev) as clk:
        for order in ("plain", "learned"):
            chk.set_launch_config(**tuned[order])
            results[order] = time_order(chk, d_edges, d_res, E, order, stream, args.steps, args.warmup, flush, dev,
                                        robot)
        chk.mlp_set_params(_mlp.init_params(1000))
        chk.set_launch_config(**tuned["learned"])
        untrained_ms = max_over_ranks(dist, time_order(chk, d_edges, d_res, E, "learned", stream, args.steps,
                                                       args.warmup, flush, dev, robot, eager_reps=0)[0],
                                      f"cuda:{dev}") / args.steps
        chk.mlp_set_params(trained_params)
    torch.cuda.synchronize()

    ms = {o: max_over_ranks(dist, results[o][0], f"cuda:{dev}") / args.steps for o in results}
    head = args.order
    value = world * N * E / (ms[head] * 1e-3)

    # Verdict agreement of the two orders (must be identical), and work counters.
    chk.set_launch_config(**tuned["plain"])
    chk.check_device(d_edges.data_ptr(), E, d_res.data_ptr(), order="plain", stream=stream.cuda_stream, robot=robot)
    chk.set_launch_config(**tuned["learned"])
    chk.check_device(d_edges.data_ptr(), E, d_res2.data_ptr(), order="learned", stream=stream.cuda_stream,
                     robot=robot)
    torch.cuda.synchronize()
    mismatch = int((d_res != d_res2).sum().item())
    verdicts = {"plain": d_res.cpu().numpy(), "learned": d_res2.cpu().numpy()}
    work = {}
    chk.set_profiling(True, counters=True)
    for order in ("plain", "learned"):
        chk.set_launch_config(**tuned[order])
        chk.check_device(d_edges.data_ptr(), E, d_res.data_ptr(), order=order, stream=stream.cuda_stream, robot=robot)
        torch.cuda.synchronize()
        c = chk.work_counters()
        work[order] = {k: v / max(c["pairs"], 1) for k, v in c.items() if k != "pairs"}
        work[order]["pairs_walked"] = c["pairs"]
    # work counters of the untrained network's learned order (the ablation)
    chk.mlp_set_params(_mlp.init_params(1000))
    chk.set_launch_config(**tuned["learned"])
    chk.check_device(d_edges.data_ptr(), E, d_res.data_ptr(), order="learned", stream=stream.cuda_stream, robot=robot)
    torch.cuda.synchronize()
    c = chk.work_counters()
    work_untrained = {k: v / max(c["pairs"], 1) for k, v in c.items() if k != "pairs"}
    chk.set_profiling(True)
    chk.mlp_set_params(trained_params)
    chk.check_device(d_edges.data_ptr(), E, d_res.data_ptr(), order="learned", stream=stream.cuda_stream, robot=robot)
    torch.cuda.synchronize()
    learned_rows = chk.last_learned_rows()
    learned_pairs = chk.last_learned_pairs()
    ranking = proposal_ranking(chk, edges, TRAIN_QUEUE_MIN_ITEMS, robot)
    proposal["uniform_samples"] = dict(chk.mlp_evaluate(edges, 1 << 20, seed=7, robot=robot),
                                       note="misprediction against the exact checker on 2^20 uniformly drawn "
                                            "(env, edge, sample) triples of the benchmark inputs")

    # e2e: the public host API (pinned host edges in, verdicts out), per step.
    h_edges = torch.from_numpy(edges).pin_memory().numpy()
    h_res = torch.empty((E, N), dtype=torch.uint8).pin_memory().numpy()
    chk.set_launch_config(**tuned[head])
    chk.check(h_edges, out=h_res, order=head, robot=robot, graph=True)
    t_e2e = []
    for _ in range(max(3, min(args.steps, 5))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        chk.check(h_edges, out=h_res, order=head, robot=robot, graph=True)
        t_e2e.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(dist, statistics.median(t_e2e), f"cuda:{dev}")
    mlp_ms, mlp_tf = mlp_roofline(chk, dev)

    if rank != 0:
        chk.close()
        return
    line = {"metric": metric_of(args.workload, N), "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms[head], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; no public dataset)",
            "config": bench_config(args.workload, N, E, world), "order": head,
            "orders": {o: {"value": world * N * E / (ms[o] * 1e-3), "ms_per_step": ms[o],
                           "launch": dict(tuned[o], graph=True), "stages_ms_per_step_eager": results[o][2],
                           "work_per_pair": work[o]} for o in results},
            "learned_over_plain": ms["plain"] / ms["learned"],
            "ablation_untrained_network": {
                "value": world * N * E / (untrained_ms * 1e-3), "ms_per_step": untrained_ms,
                "over_plain": ms["plain"] / untrained_ms, "work_per_pair": work_untrained,
                "note": "the learned pipeline with the same launch, the network at its seeded initialisation "
                        "(untrained): learned_over_plain minus this over_plain is what the training adds"},
            "verdict_mismatches_learned_vs_plain": mismatch,
            "proposal": dict(proposal, scored_segments_per_step=learned_rows, queued_pairs_per_step=learned_pairs,
                             queued_fraction=learned_pairs / float(N * E), ranking=ranking),
            # plain: steps, scan, FK (+ self-collision for row-major tables), [self,]
            # swept, check; learned adds features, MLP and ranking; its ablation
            # launches the same
            "gpu_launches": (3 * plain_launches(robot) + 2 * 3) * args.steps,
            "clocks": clk.summary()}
    line["e2e"] = {"value": world * N * E / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(edges.nbytes),
                   "d2h_bytes_per_step": int(N * E),
                   "path": "bcc_check (host edges in, host verdicts out; bcc_opts.use_graph = 1)"}
    # Roofline of the dominant kernel (environment check, plain order).  It is
    # bound by instruction issue (integer/logic and FP32 SIMT work on L2- and
    # shared-memory-resident inputs, DRAM a few per cent busy), so the roofline
    # is issue slots: achieved = warp instructions per launch (the committed ncu
    # count per pair x this launch's pairs) / the launch's CUDA-event duration,
    # peak = 148 SMs x 4 issue slots per cycle x the SM clock sampled during the
    # timed region.  The executed FP32 arithmetic is reported beside it against
    # the FMA probe's peak, and the reference's plain-order work (oracle count)
    # as the work the design avoids.
    chk_ms = statistics.mean(results["plain"][1])
    counts = committed_counts(args.workload) if (args.envs is None and args.edges is None) else None
    clocks = line["clocks"]
    sm_mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    import torch as _t
    sms = _t.cuda.get_device_properties(dev).multi_processor_count
    issue_peak = sms * 4 * sm_mhz * 1e6 / 1e9  # G warp-instructions / s
    fp32_peak = measure_fp32_peak(dev)
    ref_flops, rel_err = algorithmic_flops(envs, edges, args.flop_sample, robot)
    pairs = float(N * E)
    roof = {"bound": "issue", "unit": "G warp-instructions/s", "peak": issue_peak,
            "peak_source": "%d SMs x 4 warp-instruction issue slots per cycle x %.0f MHz (median SM clock sampled "
                           "during the timed region)" % (sms, sm_mhz),
            "kernel": "check_kernel (plain order)", "kernel_ms": chk_ms,
            "work_avoided": {"reference_plain_order_flops_per_launch": ref_flops,
                             "flop_estimate_rel_stderr": rel_err,
                             "note": "FP32 FLOPs the reference's literal plain order spends on these pairs (oracle "
                                     "count); hoisted FK and self checks, culling and the finer early exit avoid "
                                     "most of it"}}
    if counts:
        inst = counts["inst_per_pair"] * pairs
        flop = (2.0 * counts["ffma_per_pair"] + counts["fadd_per_pair"] + counts["fmul_per_pair"]) * pairs
        roof.update({"achieved": inst / (chk_ms * 1e-3) / 1e9, "frac": inst / (chk_ms * 1e-3) / 1e9 / issue_peak,
                     "traffic": counts["dram_bytes_per_pair"] * pairs,
                     "executed_warp_instructions_per_launch": inst,
                     "counts_source": "ncu sm__inst_executed.sum, smsp__sass_thread_inst_executed_op_{ffma,fadd,"
                                      "fmul}_pred_on.sum, dram__bytes_{read,write}.sum of one plain check_kernel "
                                      "launch, per pair, scaled by this launch's pairs (%s)" % COUNTS_FILE,
                     "fp32": {"achieved_tflops": flop / (chk_ms * 1e-3) / 1e12, "peak": fp32_peak,
                              "frac": flop / (chk_ms * 1e-3) / 1e12 / fp32_peak,
                              "peak_source": "FP32 FMA probe kernel measured in this run (bcc_measure_fp32_peak)"}})
        roof["work_avoided"]["factor"] = ref_flops / flop
    else:
        roof.update({"achieved": None, "frac": None, "traffic": None,
                     "note": "no committed ncu counts for this workload / size"})
    line["roofline"] = roof
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    bf16_peak = peaks.get("bf16_tflops")
    line["roofline_mlp"] = {"bound": "tensor", "achieved": mlp_tf, "peak": bf16_peak or 1590.0,
                            "unit": "TFLOP/s", "frac": mlp_tf / (bf16_peak or 1590.0),
                            "kernel": "mlp_forward_kernel (tcgen05, 4M rows)", "kernel_ms": mlp_ms,
                            "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst) of measured" if bf16_peak else
                            "fallback 1590 TFLOP/s (an earlier cuBLAS BF16 measurement on these B200s; "
                            "MEASURED_PEAKS.json absent)"}
    if not args.no_parity:
        par, ref_cuda = parity_vs_reference(envs, edges, verdicts, robot)
        if par is not None:
            line["parity"] = par
            line["reference_cuda"] = ref_cuda
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(envs, edges, robot)
    if world == 1 and args.workload == WORKLOAD and args.envs is None and args.edges is None and not args.no_others:
        others = {}
        with ClockSampler(dev) as clk2:
            for name in OTHER_WORKLOADS:
                others[name] = measure_workload(chk, name, steps=3, warmup=2, flush=flush, dev=dev,
                                                parity=not args.no_parity)
        line["other_workloads"] = dict(others, clocks=clk2.summary())
    chk.close()
    print(json.dumps(line))


def main():
    args = parse()
    world, rank, local, dist = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.profile_order:
            run_profile(args, local)
        else:
            run_ours(args, world, rank, local, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
