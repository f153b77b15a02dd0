#!/usr/bin/env python
"""Throughput of pot's per-timestep particle loop on B200.

Metric: particle-steps/s (plasma particles x base time steps; ions keep the
reference's sub-cycling, pot.c:4157-4159).  Headline workload: the
4,000,001-particle spheroid plasma of pot-spheroid.c (prolate grain of
semi-axes 0.3 / 0.1 / 0.1 Debye lengths with its axis along the flow axis x,
as the reference program has it; Te/Ti = 10, Mach-0.5 drift, B = 0.9533 T,
R = 12 Debye lengths, theta = 0.4), fast form (FP32 leaf-grouped walk, FP64
positions and push, leaf size 16, groups of 64).  Synthetic data: particles
initialised on the device by the reference's init_particles sampler with a
fixed seed.

Our arm (default):
  * value: K device-timed steps with every input resident in HBM, CUDA events
    around each step on the library's stream, L2 flushed (a 256 MiB write)
    between steps outside the timed intervals; max over ranks.  Each step is
    one replay of the library's CUDA graph of a step;
  * e2e: the drop-in call pot_gpu_move_particles on pinned host buffers in
    the reference's Particle layout (upload, step, download every step),
    wall-clock around the loop;
  * plain_fp64: the same workload with the plain FP64 form (the reference's
    arithmetic, leaf size 1);
  * roofline: the dominant kernel (the walk) against its bound, FP32
    arithmetic (flops per interaction x interactions per launch over the
    launch's CUDA-event time), with its HBM bytes beside it; the per-kernel
    events come from a second pass over the same K steps from the same
    start, with an event pair around every kernel (events cannot sit inside
    the graph);
  * kernels: every kernel's time per launch, algorithmic bytes and fraction
    of the measured HBM bandwidth;
  * cpu_baseline: the reference program itself (oracle/_ref, one core, one
    MPI rank) on a bounded sample of the same configuration.
Reference arm (--impl reference): the compiled reference on the host cores,
P processes each playing one MPI rank of a P-rank run (full tree build,
its own block of particles pushed), max over ranks per step.

Multi-GPU (--gpus N under torchrun): independent replicas, one per GPU,
different seeds, no collective in the data path (the run has a global tree
dependency and does not shard).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1 B200 vs plain GPU & CPU; batch p99 latency @1% charge err"
UNIT = "particle-steps/s"
WORKLOADS = {
    "1m": ("1m plasma: 1,000,001 particles (grain + 500,000 ions + 500,000 electrons), Te/Ti = 10, "
           "Mach-1 ion drift along x, R = 10 lambda_De, a = 0.2 lambda_De, theta = 0.5, "
           "SCEPTIC reinjection, dt = 0.005/omega_pe"),
    "4m": ("4m spheroid plasma (pot-spheroid.c): 4,000,001 particles, prolate grain 0.3/0.1/0.1 lambda_De "
           "with its axis along the flow (x, as the reference has it), Te/Ti = 10, Mach-0.5 drift, "
           "B = 0.9533 T (electron gyroradius 0.5 lambda_De), R = 12 lambda_De, theta = 0.4, SCEPTIC "
           "reinjection, dt = 0.005/omega_pe"),
    "4m_tilt": ("4m spheroid plasma with the grain tilted 30 deg to the flow (GPU only: the reference cannot "
                "tilt its grain): 4,000,001 particles, prolate grain 0.3/0.1/0.1 lambda_De, Te/Ti = 10, "
                "Mach-0.5 drift, B = 0.9533 T, R = 12 lambda_De, theta = 0.4, SCEPTIC reinjection"),
    "small": ("small plasma: 8,193 particles, Te = Ti, no flow, R = 5 lambda_De, a = 0.1 lambda_De, "
              "theta = 0.5"),
}
WORKLOAD = WORKLOADS["4m"]


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def reduce_max(x: float, device=None) -> float:
    """Max over ranks of a per-rank timing (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = "/tmp/pot_bench_clocks_%d.csv" % os.getpid()

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        try:
            os.remove(self.path)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def reference_tree_field(cfg_name: str, parts, grain, idx, xyz):
    """The reference's own field_particle_feels_at (pot.c:1696-1808) on its
    own tree built from the snapshot `parts` (reference order), for the
    targets idx at xyz; None where the compiled reference is absent."""
    from oracle.oracle import RefLib, RunParams
    from pot_b200.configs import run_params, variant
    try:
        ref = RefLib(variant(cfg_name), build=False)
    except Exception:
        return None
    p = RunParams(**run_params(cfg_name, untilted=True))
    ref.setup(p, seed=1, init=False)
    ref.set_particles(parts)
    ref.set_grain(q=int(grain["q"]), m=float(grain["m"]), tot_absor_e=int(grain["tot_absor_e"]),
                  t_steps=int(grain["t_steps"]), chi_b=float(grain["chi_b"]))
    ref.build_tree()
    hi, lo = ref.field_many(idx, xyz)
    return hi + lo


def grain_field_fp64(cfg_name: str, grain, xyz):
    """The spheroidal grain's own analytic field (pot-spheroid.c:1689-1779)
    at the points xyz, from the oracle's FP64 restatement (the spheroid is
    not a tree source, so a direct sum over the plasma leaves it out)."""
    from oracle.oracle import Oracle, RunParams
    from pot_b200.configs import run_params
    from pot_b200.gpu import PARTICLE_DTYPE
    p = RunParams(**run_params(cfg_name, N=3))
    o = Oracle(p, mode="gpu", init=False)
    parts = np.zeros(3, PARTICLE_DTYPE)
    parts["species"] = [0, 1, 2]
    parts[0]["x"], parts[0]["y"], parts[0]["z"] = grain["x"], grain["y"], grain["z"]
    o.set_particles(parts)
    o.set_grain(q=int(grain["q"]))
    return np.array([o.grain_field(*map(float, r)) for r in np.asarray(xyz)])


def direct_field_fp64(parts, grain, idx, xyz, soft, dev, grain_source=True):
    """FP64 direct sum of the field at xyz for the targets idx over every
    other particle, every pair softened as the reference's own accuracy check
    softens them (pot.c:2197-2238); torch on the GPU as the checker's
    arithmetic.  grain_source=False leaves the grain (slot 0) out of the sum
    (a spheroid, whose field is analytic)."""
    import torch
    q = np.where(parts["species"] == 0, float(grain["q"]) if grain_source else 0.0,
                 np.where(parts["species"] == 1, 1.0, -1.0))
    src = torch.tensor(np.stack([parts["x"], parts["y"], parts["z"]], 1), dtype=torch.float64, device=dev)
    qs = torch.tensor(q, dtype=torch.float64, device=dev)
    tgt = torch.tensor(np.asarray(xyz), dtype=torch.float64, device=dev)
    tid = torch.tensor(np.asarray(idx, np.int64), device=dev)
    E = torch.zeros((len(idx), 3), dtype=torch.float64, device=dev)
    n = len(parts)
    chunk = 4096
    for j0 in range(0, n, chunk):
        s = src[j0:j0 + chunk]
        d = tgt[:, None, :] - s[None, :, :]
        r2 = (d * d).sum(-1) + soft * soft
        w = qs[j0:j0 + chunk][None, :] * torch.rsqrt(r2) / r2
        jj = torch.arange(j0, j0 + s.shape[0], device=dev)
        w = w.masked_fill(tid[:, None] == jj[None, :], 0.0)
        E += (w[..., None] * d).sum(1)
    return (E * (1.6021766e-19 / (4 * 3.14159265358979 * 8.85419e-12))).cpu().numpy()


def force_accuracy(run, cfg_name: str, cfg, dev, n_targets: int = 8192):
    """Field of the fast form at n_targets sampled particles of the run's
    current state against an FP64 direct sum and against the reference's own
    tree on the same snapshot: RMS and 99th percentile of |dE| / |E_direct|."""
    parts, grain = run.download()
    rng = np.random.default_rng(12345)
    idx = np.sort(rng.choice(np.arange(1, len(parts)), n_targets, replace=False)).astype(np.uint32)
    xyz = np.stack([parts["x"][idx], parts["y"][idx], parts["z"][idx]], 1)
    run.build_tree()
    e_fast = run.field_at(idx, xyz)
    spheroid = bool(cfg.A)
    e_dir = direct_field_fp64(parts, grain, idx, xyz, cfg.soft, dev, grain_source=not spheroid)
    if spheroid:
        g = dict(grain, x=parts[0]["x"], y=parts[0]["y"], z=parts[0]["z"])
        e_dir = e_dir + grain_field_fp64(cfg_name, g, xyz)
    e_ref = reference_tree_field(cfg_name, parts, grain, idx, xyz)
    mag2 = (e_dir ** 2).sum(1)

    def stat(e):
        rel = np.sqrt(((e - e_dir) ** 2).sum(1) / mag2)
        return {"rms": float(np.sqrt(np.mean(rel ** 2))), "p99": float(np.percentile(rel, 99))}

    out = {"targets": n_targets, "state": "after the timed steps",
           "direct": "FP64, every pair softened" + (", plus the spheroid's analytic field" if spheroid else ""),
           "fast_vs_direct": stat(e_fast)}
    if e_ref is not None:
        out["reference_tree_vs_direct"] = stat(e_ref)
        rel = np.sqrt(((e_fast - e_ref) ** 2).sum(1) / (e_ref ** 2).sum(1))
        out["fast_vs_reference_tree"] = {"rms": float(np.sqrt(np.mean(rel ** 2))), "p99": float(np.percentile(rel, 99))}
    return out


def push_field_accuracy(run, cfg_name: str, cfg, dev, n_targets: int = 8192):
    """The field the fast form's push actually applied in one step, against
    an FP64 direct sum (plus the spheroid's analytic field) and against the
    reference's own tree, at the same positions: the half-drifted positions
    x0 + v0 dt / 2 of n_targets sampled electrons that the step neither
    absorbed nor reinjected.  The field comes back from the velocity change
    through the Boris step (pot.c:2475-2532): v1 = e + R(v0 + e), e = q E dt
    / (2 m), R the rotation about the field's direction by 2 atan(q B dt /
    (2 m)), so E = (2 m / (q dt)) (I + R)^-1 (v1 - R v0)."""
    P0, g0 = run.download()
    run.step(1)
    P1, _ = run.download()
    qe, me = 1.6021766e-19, 9.109383e-31
    qom = -qe / me
    dt = cfg.dt  # electrons move every step
    B = np.asarray(cfg.B, float)
    bmag = float(np.sqrt((B * B).sum()))
    R = np.eye(3)
    if bmag > 0.0:
        b = B / bmag
        ang = 2.0 * np.arctan(0.5 * dt * qom * bmag)
        K = np.array([[0.0, -b[2], b[1]], [b[2], 0.0, -b[0]], [-b[1], b[0], 0.0]])  # K v = b x v
        # rotate_vec_about_dir (coord.c:45-59): v cos + (b x v) sin + b (b.v)(1 - cos)
        R = np.cos(ang) * np.eye(3) + np.sin(ang) * K + (1.0 - np.cos(ang)) * np.outer(b, b)
    Rad = cfg.r * cfg.mpp
    moved = np.sqrt((P1["x"] - P0["x"]) ** 2 + (P1["y"] - P0["y"]) ** 2 + (P1["z"] - P0["z"]) ** 2)
    cand = np.nonzero((P0["species"] == 2) & (moved < 1e-3 * Rad))[0]
    rng = np.random.default_rng(4321)
    idx = np.sort(rng.choice(cand, min(n_targets, len(cand)), replace=False)).astype(np.uint32)
    v0 = np.stack([P0["vx"][idx], P0["vy"][idx], P0["vz"][idx]], 1)
    v1 = np.stack([P1["vx"][idx], P1["vy"][idx], P1["vz"][idx]], 1)
    e = np.linalg.solve(np.eye(3) + R, (v1 - v0 @ R.T).T).T
    E_push = e * 2.0 / (qom * dt)
    h = np.stack([P0["x"][idx] + 0.5 * dt * P0["vx"][idx], P0["y"][idx] + 0.5 * dt * P0["vy"][idx],
                  P0["z"][idx] + 0.5 * dt * P0["vz"][idx]], 1)
    spheroid = bool(cfg.A)
    e_dir = direct_field_fp64(P0, g0, idx, h, cfg.soft, dev, grain_source=not spheroid)
    if spheroid:
        g = dict(g0, x=P0[0]["x"], y=P0[0]["y"], z=P0[0]["z"])
        e_dir = e_dir + grain_field_fp64(cfg_name, g, h)
    e_ref = reference_tree_field(cfg_name, P0, g0, idx, h)
    mag2 = (e_dir ** 2).sum(1)

    def stat(ev):
        rel = np.sqrt(((ev - e_dir) ** 2).sum(1) / mag2)
        return {"rms": float(np.sqrt(np.mean(rel ** 2))), "p99": float(np.percentile(rel, 99))}

    out = {"targets": int(len(idx)), "state": "one step after the timed steps",
           "field": "recovered from the push's velocity change through the Boris step",
           "direct": "FP64, every pair softened" + (", plus the spheroid's analytic field" if spheroid else ""),
           "push_vs_direct": stat(E_push)}
    if e_ref is not None:
        out["reference_tree_vs_direct"] = stat(e_ref)
    return out


def cpu_baseline_reference(cfg_name: str):
    """The reference program (compiled from its own sources, one MPI rank on
    one core) on a bounded sample of the same configuration.

    Up to 1.5M particles the sample is one whole step.  Above that a whole
    step takes minutes on one core, so the sample is the reference's own
    16-rank decomposition seen from its last rank (pot.c:2936-2998 blocks,
    reference order grain, ions, electrons: the last block is all
    electrons): its build_tree alone, then one step of that rank (the tree
    again plus its block pushed).  The one-core step is the tree plus every
    due electron at the block's push rate."""
    from oracle.oracle import RefLib, RunParams
    from pot_b200.configs import run_params, variant
    p = RunParams(**run_params(cfg_name, untilted=True))
    n_plasma = p.N - 1
    try:
        ref = RefLib(variant(cfg_name), build=False)
    except Exception:
        ref = None
    if ref is not None and p.N <= 1_500_000:
        t0 = time.perf_counter()
        ref.setup(p, seed=1)
        t_init = time.perf_counter() - t0
        t0 = time.perf_counter()
        ref.step()
        t_step = time.perf_counter() - t0
        return {"value": n_plasma / t_step, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "one step (t = 1: tree over %d particles, %d electrons pushed) of the %s config by the "
                          "reference pot.c compiled with gcc -O2 and a single-rank MPI stand-in, after its own "
                          "init_particles (%.1f s); step took %.1f s" % (p.N, n_plasma // 2, cfg_name, t_init,
                                                                         t_step)}
    if ref is not None:
        P = 16
        t0 = time.perf_counter()
        ref.setup(p, seed=1, nprocs=P, rank=P - 1)
        t_init = time.perf_counter() - t0
        t0 = time.perf_counter()
        ref.build_tree()
        t_tree = time.perf_counter() - t0
        t0 = time.perf_counter()
        ref.step()
        t_rank = time.perf_counter() - t0
        # the last block [lo, N): init_particles lays out each block as its
        # ions then its electrons (pot.c:908-930); at t = 1 only electrons
        # are due
        lo = (P - 1) * (p.N // P)
        sp = ref.particles()["species"]
        e_block = int((sp[lo:] == 2).sum())
        n_e = int((sp == 2).sum())
        t_push = max(t_rank - t_tree, 1e-9)
        t_one = t_tree + t_push * n_e / max(e_block, 1)
        return {"value": n_plasma / t_one, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "the reference (pot-spheroid.c / pot.c, gcc -O2, single-rank MPI stand-in) as the last "
                          "rank of an %d-rank run of the %s config (t = 1, after its own init_particles, %.1f s): "
                          "build_tree over %d particles %.2f s, then one step of that rank %.2f s (tree + its %d "
                          "electrons pushed); one-core step = tree + all %d electrons at that push rate = %.1f s"
                          % (P, cfg_name, t_init, p.N, t_tree, t_rank, e_block, n_e, t_one)}
    from oracle.oracle import Oracle
    o = Oracle(p, mode="reference", seed=1, sceptic=variant(cfg_name).endswith("sceptic"))
    t0 = time.perf_counter()
    o.step()
    t_step = time.perf_counter() - t0
    return {"value": n_plasma / t_step, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "one step of the %s config by the C restatement (reference not built here)" % cfg_name}


def _ref_rank_worker(args):
    cfg_name, nprocs, rank, n_steps, budget_s, q = args
    from oracle.oracle import RefLib, RunParams
    from pot_b200.configs import run_params, variant
    p = RunParams(**run_params(cfg_name, untilted=True))
    ref = RefLib(variant(cfg_name), build=False)
    ref.setup(p, seed=1, nprocs=nprocs, rank=rank)
    times = []
    start = time.perf_counter()
    # the run is a bounded sample: steps stop at n_steps or once budget_s of
    # stepping has passed (at least two steps)
    for k in range(n_steps):
        if k >= 2 and time.perf_counter() - start > budget_s:
            break
        t0 = time.perf_counter()
        ref.step()
        times.append(time.perf_counter() - t0)
    q.put((rank, times))


def run_reference_arm(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    import multiprocessing as mp
    try:
        import psutil
        mem_gb = psutil.virtual_memory().available / 2 ** 30
    except Exception:
        mem_gb = 64.0
    from pot_b200.configs import CONFIGS
    N = CONFIGS[args.config]["N"]
    per_proc_gb = N * (56 * 2 + 9 * 130 + 48 + 24) / 2 ** 30 + 0.1
    cores = len(os.sched_getaffinity(0))
    P = max(1, min(cores, int(mem_gb * 0.6 / per_proc_gb), 64))
    # each step is a bounded sample: at most a few minutes for the whole run
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    n = args.warmup + args.steps
    budget_s = 150.0
    procs = [ctx.Process(target=_ref_rank_worker, args=((args.config, P, r, n, budget_s, q),)) for r in range(P)]
    for pr in procs:
        pr.start()
    res = {}
    import queue as _queue
    failed = None
    while len(res) < P and failed is None:
        try:
            r, times = q.get(timeout=10)
            res[r] = times
        except _queue.Empty:
            dead = [pr.exitcode for pr in procs if pr.exitcode not in (None, 0)]
            if dead:
                failed = "a reference rank exited with status %d" % dead[0]
    for pr in procs:
        if failed is not None and pr.is_alive():
            pr.terminate()
        pr.join()
    if failed is not None:
        print(json.dumps({"impl": "reference", "unavailable": failed}), flush=True)
        return 1
    # every rank ran the same steps up to its budget; the common prefix, less
    # the warm-up steps (at most half of it), is timed
    common = min(len(res[r]) for r in range(P))
    w = min(args.warmup, common // 2)
    per_step = [max(res[r][k] for r in range(P)) for k in range(common)][w:]
    timed = len(per_step)
    t = sum(per_step)
    value = (N - 1) * timed / t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / timed,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64/x87",
            "data": "synthetic", "config": {"workload": WORKLOADS.get(args.config, args.config), "N": N,
                                            "reference_axis": "x (pot-spheroid.c's spheroid axis; the reference "
                                                              "cannot tilt its grain)"
                                            if CONFIGS[args.config].get("A") else None},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": P, "kind": "reference",
                             "sample": "%d processes, each one MPI rank of a %d-rank run of the reference pot.c "
                                       "(gcc -O2, single-rank MPI stand-in): full tree build plus its own block "
                                       "of ~%d particles per step; step time = max over ranks; no MPI "
                                       "communication counted; %d timed steps after %d warm-up (at most %.0f s "
                                       "of stepping per rank)" % (P, P, N // P, timed, w, budget_s)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_batches(args, device):
    """The batched sweep and the serving loop (pot_b200/potserve), short
    versions sized so that most runs converge inside them: a sweep of
    --batch-runs runs of 16k-64k particles and a serving window of Poisson
    arrivals (20 per second for --serve-seconds, 8k-128k particles), each run
    to a converged charge (the 500-step moving mean changing by under 0.5 %)
    or --batch-steps steps.  Packed launches, autotuned group and leaf sizes,
    the sampler's edge-potential cap on (POT_OPT_CHI_CAP).  The full-length
    sweep (16k-256k) and serving load (8k-1M) are separate invocations."""
    from pot_b200 import build as gpu_build
    try:
        exe = os.path.join(os.path.dirname(gpu_build.HOST_BIN), "potserve")
        if not os.path.exists(exe):
            gpu_build.build_host()
    except Exception as e:  # no compiler and no binary
        return {"unavailable": str(e)}
    out = {}
    common = ["--max-steps", str(args.batch_steps), "--tune", "--device", str(device)]
    runs = [("sweep", ["--mode", "sweep", "--runs", str(args.batch_runs), "--nmin", "16000", "--nmax", "64000"]),
            ("serve", ["--mode", "serve", "--rate", "20", "--duration", str(args.serve_seconds), "--nmin", "8000",
                       "--nmax", "128000", "--bmax", "1.0"])]
    for name, extra in runs:
        try:
            p = subprocess.run([exe] + extra + common, capture_output=True, text=True, timeout=600)
            out[name] = json.loads(p.stdout) if p.returncode == 0 else {"error": p.stderr[-400:]}
        except Exception as e:
            out[name] = {"error": str(e)}
    return out


def kernel_table(kt, N, pushes, hbm_peak):
    """Per-kernel time per launch, algorithmic bytes per launch and the
    fraction of the measured HBM bandwidth they represent.  Algorithmic
    bytes count each array a kernel must read or write once: keys (FP64
    position in, 64-bit key and 32-bit slot out), the sort's histogram (keys
    in) and each onesweep pass (key and slot in and out), the reorder
    (gather of position, velocity and identity; write of the same plus FP64
    and FP32 sources and a due flag), the compaction (due flags in, list
    and prefix out), the fast moments (FP32 sources in, per-particle FP64
    prefix sums out and read back per cell) and the walk (FP64 state of each
    pushed particle in and out).  Kernels bound by latency or L2 (tree
    build, groups, reinjection, grain update) get none."""
    per_particle = {"keys": 32 + 12, "sort_hist": 8, "sort_pass": 24, "reorder": 72 + 117, "compact": 1 + 8,
                    "tree_moments": 16 + 40 + 40}
    out = {}
    for name, (ms, n) in sorted(kt.items(), key=lambda kv: -kv[1][0]):
        per = ms / max(n, 1)
        if name.startswith("walk_push") or name.startswith("walk_half2"):
            b = 96.0 * pushes
        elif name in per_particle:
            b = per_particle[name] * float(N)
        else:
            b = None
        e = {"ms": round(per, 4), "launches": n, "alg_bytes": b}
        if b:
            gbs = b / (per / 1e3) / 1e9
            e["hbm_gbs"] = round(gbs, 1)
            e["hbm_frac"] = round(gbs / hbm_peak, 4)
        out[name] = e
    return out


def roofline(kernel, interactions, far_cells, pushes, launch_s, clk, alg_bytes, hbm_achieved, hbm_peak, peak_kind,
             traffic, share, timing):
    """The dominant kernel against its bound.  The fast walk is bound by
    FP32 arithmetic and instruction issue, not HBM.  Its arithmetic per
    launch: 17 FP32 flops (and one reciprocal square root) per
    target-source interaction, 60 per far cell expanded about its group's
    centre (field, first and second derivatives, once per group) and 45 per
    push (the expansion evaluated at the target), counts from the device
    counters, over the launch's CUDA-event time; against 148 SMs x 128 FP32
    lanes x 2 flops x the median SM clock sampled during the timed region
    (a nominal peak: no measured FP32 figure exists).  Its HBM figures (96 B
    per push: the FP64 state read and written) sit beside it; `traffic` is
    the DRAM bytes of one launch from an ncu capture of the same workload."""
    mhz = (clk or {}).get("sm_mhz") or 1965.0
    out = {"kernel": kernel, "ms_per_launch": launch_s * 1e3, "share_of_step": share, "timing": timing,
           "alg_bytes_per_launch": alg_bytes, "traffic": traffic,
           "hbm": {"achieved": hbm_achieved, "peak": hbm_peak, "peak_kind": peak_kind, "unit": "GB/s",
                   "frac": hbm_achieved / hbm_peak}}
    if interactions and kernel.startswith("walk_push") and launch_s:
        flops = interactions * 17.0 + (far_cells * 60.0 + pushes * 45.0 if far_cells else 0.0)
        achieved = flops / launch_s / 1e12
        peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
        out.update({"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                    "peak_kind": "nominal FP32 at the sampled SM clock (%.0f MHz)" % mhz,
                    "flop_per_interaction": 17, "interactions_per_launch": interactions,
                    "far_cells_per_launch": far_cells, "flop_per_far_cell": 60, "flop_per_push_expansion": 45})
    else:
        out.update({"bound": "hbm", "achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s",
                    "frac": hbm_achieved / hbm_peak, "peak_kind": peak_kind})
    return out


def time_config(name, stream, dev, flush, steps=10, warmup=3, plain_steps=3):
    """Device-timed steps of another configuration, fast form and plain
    FP64 form, with the same event / L2-flush discipline as the main line."""
    import torch

    from pot_b200.configs import CONFIGS, run_config
    from pot_b200.gpu import Run

    cfgd = CONFIGS[name]
    cfg = run_config(name)
    out = {"workload": WORKLOADS.get(name, name), "N": cfg.N, "steps": steps}

    def timed(run, k):
        run.init_particles()
        for _ in range(warmup):
            run.step_async(1)
        run.sync()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        torch.cuda.synchronize(dev)
        for a, b in ev:
            a.record(stream)
            run.step_async(1)
            b.record(stream)
            flush.zero_()
        torch.cuda.synchronize(dev)
        st = run.step(0)
        return sum(a.elapsed_time(b) for a, b in ev) / k, st

    group = cfgd.get("group_size", 32)
    with Run(cfg, form="fast", leaf_size=cfgd["leaf_size"], group_size=group, seed=cfgd.get("seed", 1),
             stream=stream.cuda_stream, device=dev.index) as run:
        ms, st = timed(run, steps)
    out["fast"] = {"value": (cfg.N - 1) / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
                   "form": "fast FP32 walk / FP64 state, leaf %d, groups of %d" % (cfgd["leaf_size"], group),
                   "status": st["status"]}
    with Run(cfg, form="plain", seed=cfgd.get("seed", 1), stream=stream.cuda_stream, device=dev.index) as run:
        msp, stp = timed(run, plain_steps)
    out["plain_fp64"] = {"value": (cfg.N - 1) / (msp / 1e3), "unit": UNIT, "ms_per_step": msp,
                         "steps": plain_steps, "form": "plain FP64, leaf 1", "status": stp["status"]}
    out["fast_over_plain"] = msp / ms
    return out


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from pot_b200.configs import CONFIGS, run_config
    from pot_b200.gpu import PARTICLE_DTYPE, Run

    ws, rank, local = dist_env()
    if ws > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # a dedicated stream: the library launches on it and the events are recorded on it
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0
    cfgd = CONFIGS[args.config]
    cfg = run_config(args.config, N=args.particles or None)
    N = cfg.N
    n_plasma = N - 1
    hbm_peak, peak_kind = peaks()

    group = args.group or cfgd.get("group_size", 32)
    seed0 = cfgd.get("seed", 1)
    flush = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device=dev)

    def timed_region(r, per_step_stats=False):
        """args.steps steps of r, each between CUDA events on the library's
        stream, L2 flushed after each; barrier + synchronize on both sides.
        per_step_stats: read each step's statistics after it (a host wait
        per step: the instrumented pass only)."""
        for _ in range(args.warmup):
            r.step_async(1)
        r.sync()
        r.reset_kernel_times()
        l0 = r.launch_count()
        r.step(0)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        clocks = Clocks(local)
        clocks.start()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        sums = {"interactions": 0, "n_pushed": 0, "n_groups": 0, "far_cells": 0}
        for k in range(args.steps):
            ev[k][0].record(stream)
            r.step_async(1)
            ev[k][1].record(stream)
            flush.zero_()
            if per_step_stats:
                stk = r.step(0)
                for key in sums:
                    sums[key] += int(stk.get(key) or 0)
        torch.cuda.synchronize(dev)
        if ws > 1:
            dist.barrier()
        clk_ = clocks.stop()
        r.sync()
        t = sum(a.elapsed_time(b) for a, b in ev)
        stl = r.step(0)
        if per_step_stats:
            stl = dict(stl, **{"sum_" + key: v for key, v in sums.items()})
        return t, r.launch_count() - l0, stl, clk_

    def make_run(timing):
        r = Run(cfg, form=args.form, leaf_size=args.leaf or cfgd["leaf_size"], group_size=group, seed=seed0 + rank,
                device=local, stream=stream.cuda_stream, timing=timing)
        r.init_particles()
        return r

    # the measured run: each step one CUDA-graph replay, no instrumentation
    run = make_run(False)
    t_ms, launches, st, clk = timed_region(run)
    t_ms = reduce_max(t_ms, dev)
    value = n_plasma * ws * args.steps / (t_ms / 1e3)
    # the same steps from the same start once more with a CUDA event pair
    # around every kernel: the per-kernel times behind the roofline
    runk = make_run(True)
    tk_ms, _, stk, _ = timed_region(runk, per_step_stats=True)
    kt = runk.kernel_times()
    runk.close()

    # dominant kernel: its time per launch and algorithmic bytes
    dom = max(kt.items(), key=lambda kv: kv[1][0])
    dom_name, (dom_ms, dom_n) = dom
    n_e = n_plasma - (N - 1) // 2
    tss_ion = int((cfg.Te * 1836.15 / cfg.Ti) ** 0.5)
    pushes_per_step = n_e + ((N - 1) // 2) / tss_ion  # average due particles per step
    per_launch_s = dom_ms / dom_n / 1e3
    kernels = kernel_table(kt, N, pushes_per_step, hbm_peak)
    alg_bytes = kernels[dom_name]["alg_bytes"] or 0.0
    achieved = alg_bytes / per_launch_s / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            with open(tpath) as f:
                tj = json.load(f)
            if tj.get("workload") == args.config and not args.particles:
                traffic = tj.get(dom_name)
        except Exception:
            traffic = None
    # interactions, far cells and pushes per walk launch, averaged over the
    # instrumented pass's steps
    inter = stk["sum_interactions"] / args.steps if stk.get("sum_interactions") else st["interactions"]
    far = stk.get("sum_far_cells", 0) / args.steps
    pushes_launch = stk.get("sum_n_pushed", 0) / args.steps

    # plain FP64 form on the same workload (fewer steps: it is the slow form)
    plain = None
    if args.plain_steps > 0:
        runp = Run(cfg, form="plain", seed=seed0 + rank, device=local, stream=stream.cuda_stream, timing=False)
        runp.init_particles()
        runp.step_async(1)
        runp.sync()
        evp = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.plain_steps)]
        torch.cuda.synchronize(dev)
        for k in range(args.plain_steps):
            evp[k][0].record(stream)
            runp.step_async(1)
            evp[k][1].record(stream)
            flush.zero_()
        torch.cuda.synchronize(dev)
        runp.sync()
        tp = sum(a.elapsed_time(b) for a, b in evp)
        plain = {"value": n_plasma * args.plain_steps / (tp / 1e3), "unit": UNIT,
                 "ms_per_step": tp / args.plain_steps, "steps": args.plain_steps, "form": "plain FP64, leaf 1",
                 "fast_over_plain": (tp / args.plain_steps) / (t_ms / args.steps)}
        runp.close()

    # end to end: drop-in call on pinned host buffers
    host = torch.empty(N * PARTICLE_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    parts = host.numpy().view(PARTICLE_DTYPE)
    P, g = run.download()
    parts[:] = P
    grain = g
    run.move_particles(parts, grain)  # warm
    # records the call copies back: the grain's and the reference-index range
    # of the species due at step t (host arithmetic, for the byte count only)
    sp = parts["species"]
    span = {s_: (int(np.flatnonzero(sp == s_)[0]), int(np.flatnonzero(sp == s_)[-1])) for s_ in (0, 1, 2)
            if (sp == s_).any()}
    tss = {0: tss_ion * int((0.1 * 1.67e-12 / (1836.15 * 9.109383e-31)) ** 0.5), 1: tss_ion, 2: 1}

    def d2h_records(t):
        due = [span[s_] for s_ in span if t % tss[s_] == 0]
        lo, hi = min(a for a, _ in due), max(b for _, b in due)
        return (hi - lo + 1) + (1 if lo > 0 else 0)
    t_first = int(grain["t_steps"]) + 1
    d2h_rec = sum(d2h_records(t_first + k) for k in range(args.e2e_steps))
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        grain, _ = run.move_particles(parts, grain)
    torch.cuda.synchronize(dev)
    t_e2e = time.perf_counter() - t0
    e2e = {"value": n_plasma * args.e2e_steps / t_e2e, "unit": UNIT,
           "h2d_bytes_per_step": int(N * PARTICLE_DTYPE.itemsize + 96),
           "d2h_bytes_per_step": int(d2h_rec * PARTICLE_DTYPE.itemsize / args.e2e_steps + 8 + 88),
           "steps": args.e2e_steps, "first_step": t_first,
           "timing": "wall clock around pot_gpu_move_particles calls: the whole Particle array uploaded, the "
                     "grain's record and the range of the particles due copied back"}
    if ws > 1:
        e2e["value"] = n_plasma * ws * args.e2e_steps / reduce_max(t_e2e, dev)

    cpu = None
    accuracy = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        # the reference leg: the reference's own step for the CPU baseline, and
        # its own tree for the force comparison
        cpu = cpu_baseline_reference(args.config)
        accuracy = force_accuracy(run, args.config, cfg, dev)
        accuracy["push"] = push_field_accuracy(run, args.config, cfg, dev)

    batch = None
    if ws == 1 and args.batch_runs > 0:
        batch = run_batches(args, local)

    extra = {}
    for name in ([] if ws > 1 else [c for c in args.extra_config.split(",") if c and c not in ("none", args.config)]):
        extra[name] = time_config(name, stream, dev, flush, steps=min(args.steps, 10), warmup=3,
                                  plain_steps=min(args.plain_steps, 3) or 2)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 force / f64 state", "data": "synthetic",
            "config": {"workload": WORKLOADS.get(args.config, args.config), "N": N, "form": args.form,
                       "leaf_size": args.leaf or cfgd["leaf_size"],
                       "group_size": group,
                       "l2": "flushed between timed steps (256 MiB write outside the events)",
                       "parallelism": "replicas" if ws > 1 else "1 GPU"},
            "roofline": roofline(dom_name, inter, far, pushes_launch, per_launch_s, clk, alg_bytes, achieved,
                                 hbm_peak, peak_kind, traffic, dom_ms / tk_ms if tk_ms else None,
                                 "per-kernel CUDA events in a second, instrumented pass over the same %d steps "
                                 "(%.4f ms per step with the events)" % (args.steps, tk_ms / args.steps)),
            "interactions_per_s": (inter * ws / (t_ms / args.steps / 1e3)) if inter else None,
            "interactions_per_push": (stk["sum_interactions"] / stk["sum_n_pushed"])
            if stk.get("sum_n_pushed") else None,
            "far_cells_per_group": (stk["sum_far_cells"] / stk["sum_n_groups"]) if stk.get("sum_n_groups") else None,
            "kernels": kernels,
            "gpu_launches": launches, "clocks": clk, "plain_fp64": plain, "e2e": e2e, "cpu_baseline": cpu,
            "walk_stack_max": st.get("stack_max"),
            "targets_per_group": (stk["sum_n_pushed"] / stk["sum_n_groups"]) if stk.get("sum_n_groups") else None,
            "force_accuracy": accuracy, "extra_configs": extra or None,
            "batch": batch,
            "status": st["status"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    run.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", default="4m")
    ap.add_argument("--form", choices=("fast", "plain"), default="fast")
    ap.add_argument("--leaf", type=int, default=0)
    ap.add_argument("--group", type=int, default=0, help="targets per warp group (32 or 64; default per config)")
    ap.add_argument("--particles", type=int, default=0,
                    help="override N (same domain and flags): a smaller case of the same kernels for profiling")
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-runs", type=int, default=32,
                    help="runs in the short batched sweep (0 to skip the batch and serving measurements)")
    ap.add_argument("--batch-steps", type=int, default=4000, help="step cap per run in the short batch measurements")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="arrival window of the short serving run")
    ap.add_argument("--extra-config", default="4m_tilt,1m",
                    help="also time these configurations (comma-separated; fast and plain FP64 form, N=1 only) "
                         "into the line's extra_configs; 'none' to skip")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
