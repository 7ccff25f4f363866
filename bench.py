#!/usr/bin/env python
"""Benchmark of the LOD diffusion-decay step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 256^3 voxels x 8 substrates, dt = 0.01 min, dx = 20 um, D and
lambda log-uniform in [1e2, 1e5] / [1e-3, 1] (seeded), U[0,1) field, no
Dirichlet, no agents -- the configuration the FP32 >= 70 % HBM-roofline
target is quoted on. Metric: voxel*substrate updates per second per LOD step
(V*S*K / t). A "step" is one full LOD step (x, y and z Thomas sweeps with the
fused Dirichlet), replayed from a CUDA graph. The 537 MB FP32 field is larger
than the 126 MB L2, so no flush is needed between steps.

Multi-GPU: the path does not shard (one grid per GPU); N ranks run N
independent replicas ("replicas only"), timed with CUDA events and reduced as
the max over ranks. `--impl reference` times the reference's own CPU solver
(oracle/_ref, compiled from the reference sources) on rank 0.

One JSON line is printed by rank 0.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
NX = NY = NZ = 256  # the benchmark grid; --grid / --substrates resize it for profiling small cases
S = 8
DT = 0.01
DX = 20.0
SEED = 2026
UNIT = "voxel*substrate updates/s"


def metric_name():
    return f"voxel*substrate updates/s per LOD step ({NX}^3 voxels x {S} substrates)"


def load_bfb():
    pkg = ROOT / "biofvm-b_b200"
    spec = importlib.util.spec_from_file_location("biofvm_b_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["biofvm_b_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def coefficients():
    rng = np.random.default_rng(SEED)
    D = np.exp(rng.uniform(np.log(1e2), np.log(1e5), S))
    lam = np.exp(rng.uniform(np.log(1e-3), np.log(1.0), S))
    return D, lam, rng


def initial_field(rng):
    return rng.random((NX, NY, NZ, S))


def config(extra=None):
    c = {"workload": f"LOD diffusion-decay step, {NX}^3 voxels x {S} substrates, dt={DT}, dx={DX}, "
                     "no Dirichlet, no agents",
         "grid": [NX, NY, NZ], "substrates": S, "dt": DT,
         "l2": f"inputs larger than L2 (field {NX * NY * NZ * S * 4 / 1e6:.0f} MB FP32 / "
               f"{NX * NY * NZ * S * 8 / 1e6:.0f} MB FP64 > 126 MB)",
         "parallelism": "replicas only (one grid per GPU)"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        self.proc.wait()
        rows = [r.split(",") for r in Path(self.path).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        j = json.loads(p.read_text())
        return float(j["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, STREAM-style copy)"
    return 6650.0, "fallback (6.65 TB/s)"


def ncu_traffic(kernel_key):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    j = json.loads(p.read_text())
    v = j.get(kernel_key)
    return None if v is None else float(v)


# ---------------------------------------------------------------------------
# CPU baselines (test infrastructure under oracle/, used only here)
# ---------------------------------------------------------------------------
def cpu_reference_run(max_seconds, min_steps=1, steps=None, warmup=1):
    """Time the reference's own CPU solver (oracle/_ref) on the workload, after
    `warmup` untimed steps (the first computes the Thomas factors).
    Returns (updates/s, steps timed, threads, solver name, seconds)."""
    sys.path.insert(0, str(ROOT))
    from oracle.oracle import REF_SO, RefEnv, RefLib
    if not REF_SO.exists():
        return None
    ref = RefLib()
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    ref.lib.ref_set_threads(threads)
    D, lam, rng = coefficients()
    rho0 = initial_field(rng)
    best = None
    for solver, name in ((0, "LOD_3D"), (1, "LOD_3D_AVX256D")):
        e = RefEnv(ref, (0, 0, 0, NX * DX, NY * DX, NZ * DX), DX, D, lam)
        e.set_field(rho0)
        e.set_dirichlet([0] * S)
        e.set_solver(solver)
        e.step(DT, max(1, warmup))  # untimed; the first call computes the Thomas factors
        t0 = time.perf_counter()
        n = 0
        while True:
            e.step(DT, 1)
            n += 1
            el = time.perf_counter() - t0
            if steps is not None and n >= steps:
                break
            if max_seconds is not None and n >= min_steps and el >= max_seconds:
                break
        rate = NX * NY * NZ * S * n / el
        e.close()
        del e
        if best is None or rate > best[0]:
            best = (rate, n, threads, name, el)
    return best


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), for the baseline's record."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_port_run(max_seconds):
    """Fallback when the reference is not built: our oracle port, 1 thread,
    on a 64^3 x 8 sample of the workload."""
    sys.path.insert(0, str(ROOT))
    from oracle.oracle import Oracle
    o = Oracle()
    D, lam, rng = coefficients()
    rho = rng.random((64, 64, 64, S))
    t0 = time.perf_counter()
    n = 0
    while True:
        rho = o.lod_steps(rho, DT, DX, D, lam, 1)
        n += 1
        if time.perf_counter() - t0 >= max_seconds:
            break
    el = time.perf_counter() - t0
    return 64 ** 3 * S * n / el, n


# ---------------------------------------------------------------------------
# the uneven ensemble: 256 independent microenvironments
# ---------------------------------------------------------------------------
ENSEMBLE_N = 256
ENSEMBLE_SEED = 4


def ensemble_specs(n=ENSEMBLE_N, seed=ENSEMBLE_SEED):
    """Per-instance parameters: grid edges U{32..160} per axis (non-cubic),
    1-6 substrates with D and lambda log-uniform in [1e2, 1e5] / [1e-3, 1],
    0-20k agents, Dirichlet 38.0 on the x faces for substrate 0. Each
    instance's field and agents come from its own seed, so every rank builds
    any instance identically without communicating."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        shape = tuple(int(v) for v in rng.integers(32, 161, 3))
        S_i = int(rng.integers(1, 7))
        D = np.exp(rng.uniform(np.log(1e2), np.log(1e5), S_i))
        lam = np.exp(rng.uniform(np.log(1e-3), np.log(1.0), S_i))
        specs.append({"shape": shape, "S": S_i, "D": D, "lam": lam, "agents": int(rng.integers(0, 20001)),
                      "seed": seed * 100_000 + i})
    return specs


def build_instance(bfb, spec, precision, device):
    rng = np.random.default_rng(spec["seed"])
    shape, S_i = spec["shape"], spec["S"]
    env = bfb.Env(shape, S_i, dx=DX, precision=precision, device=device)
    env.set_coefficients(spec["D"], spec["lam"])
    env.set_field(rng.random((*shape, S_i)))
    fm = np.zeros((6, S_i), np.uint8)
    fm[0:2, 0] = 1
    act = np.zeros(S_i, np.uint8)
    act[0] = 1
    env.set_dirichlet_uniform(act, np.full(S_i, 38.0), face_mask=fm)
    na = spec["agents"]
    if na:
        box = np.array(shape) * DX
        sec, upt, sat = np.exp(rng.uniform(np.log(1e-2), np.log(10.0), (3, na, S_i)))
        env.set_agents(rng.random((na, 3)) * box, np.full(na, 4.0 / 3.0 * np.pi * 125.0), sec, upt, sat, DT)
    return env


BATCH_MODE_NAMES = {0: "persistent", 1: "staged", 2: "graph"}


def time_ensemble(bfb, envs, K, stream):
    """Device time per step of the envs stepped together (bfb_batch_simulate,
    in the mode and launch shape bfb_batch_autotune picks, and in each mode
    at its default shape) and one by one (bfb_batch_simulate_loop), CUDA
    events on one stream. The autotuner restores every field it advances."""
    import torch
    flags = bfb.STEP_DIFFUSION | bfb.STEP_CELLS
    batch = bfb.Batch(envs)
    batch.set_stream(stream.cuda_stream)

    def timed(run):
        run(DT, 3, flags)  # warm-up (graph captures)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run(DT, K, flags)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / K

    out = {"modes": {}}
    for mode in (1, 0, 2):
        batch.set_mode(mode)
        out["modes"][BATCH_MODE_NAMES[mode]] = timed(batch.simulate)
    tuned, _ = batch.autotune(DT, flags, trials=2)
    out["tuned"] = {"mode": BATCH_MODE_NAMES[batch.mode], "warps_per_cta": tuned[0], "tiles_per_item": tuned[1]}
    out["batch"] = timed(batch.simulate)
    out["loop"] = timed(batch.simulate_loop)
    batch.synchronize()
    batch.close()
    return out


# ---------------------------------------------------------------------------
# collectives between ranks: torch.distributed (NCCL on GPUs, gloo in the CPU
# tests); each is a no-op in one process. The library's own ranks.py holds
# only the partition of an ensemble's instances.
# ---------------------------------------------------------------------------
def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def rank_barrier(device=None):
    """Barrier across ranks (a no-op in one process), then a device sync."""
    import torch
    dist = _dist()
    if dist is not None:
        dist.barrier()
    if device is not None and device.type == "cuda":
        torch.cuda.synchronize(device)


def _all_reduce_scalar(x, op, device):
    import torch
    dist = _dist()
    if dist is None:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, device=None):
    """The maximum of x over all ranks: the timed region of a multi-GPU run is the slowest rank's."""
    import torch.distributed as dist
    return _all_reduce_scalar(x, dist.ReduceOp.MAX, device)


def sum_over_ranks(x, device=None):
    import torch.distributed as dist
    return _all_reduce_scalar(x, dist.ReduceOp.SUM, device)


def gather_by_instance(local_ids, local_values, n_instances, width, device=None):
    """Every rank receives the [n_instances, width] array of per-instance
    values (per-substrate checksums, for example), each row filled by the rank
    that owns the instance; rows no rank owns stay 0. One all-reduce."""
    import torch
    buf = torch.zeros((n_instances, width), dtype=torch.float64, device=device)
    for i, v in zip(local_ids, local_values):
        row = torch.as_tensor(np.asarray(v, dtype=np.float64).reshape(-1)[:width], device=device)
        buf[i, :row.numel()] = row
    dist = _dist()
    if dist is not None:
        dist.all_reduce(buf, op=dist.ReduceOp.SUM)  # every row has exactly one owner
    return buf.cpu().numpy()


# ---------------------------------------------------------------------------
def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def run_reference_arm(args):
    rank, world, _ = dist_setup(args)
    if rank != 0:
        return 0
    warm = max(args.warmup, 1)
    # each solver: W untimed steps (the first sets up the factors), then up to
    # K steps or args.ref_seconds of timing, whichever comes first (a bounded sample)
    r = cpu_reference_run(args.ref_seconds, min_steps=1, steps=args.steps, warmup=warm)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref not built "
                          "(it is compiled from the reference sources by `make -C oracle ref`)"}))
        return 0
    rate, n, threads, name, el = r
    line = {
        "impl": "reference", "metric": metric_name(), "value": rate, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": warm, "ms_per_step": el / n * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded U[0,1) field, log-uniform D/lambda)",
        "config": config(),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference", "cpu": cpu_model(),
                         "solver": name, "threads": threads, "ranks": "1 rank x N threads (MPI unavailable)",
                         "sample": f"{n} of the {args.steps} requested full {NX}^3x{S} FP64 steps (capped at "
                                   f"{args.ref_seconds:.0f} s) after {warm} untimed steps (the first sets up the factors), "
                                   "best of LOD_3D / AVX256D"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_our_arm(args):
    import torch
    rank, world, local = dist_setup(args)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    bfb = load_bfb()
    warm = max(args.warmup, 3)
    K = args.steps
    V = NX * NY * NZ
    D, lam, rng = coefficients()
    rho0 = initial_field(rng)

    dev = torch.device("cuda", local)

    def barrier():
        rank_barrier(dev)

    def slowest(x):
        return max_over_ranks(x, dev)

    results = {}
    stream = torch.cuda.Stream()
    for prec, name in ((bfb.FP32, "fp32"), (bfb.FP64, "fp64")):
        env = bfb.Env((NX, NY, NZ), S, dx=DX, precision=prec, device=local)
        env.set_coefficients(D, lam)
        env.set_field(rho0)
        env.set_stream(stream.cuda_stream)
        if args.no_autotune:  # the library's default launch shapes (profiling runs: ncu distorts the tuner's timing)
            tuned = env.get_tuning()
        else:
            tuned, _ = env.autotune(DT, trials=3)  # launch shapes chosen by the library's autotuner
        env.simulate(DT, warm, bfb.STEP_DIFFUSION)
        barrier()
        clocks = Clocks(local)
        if name == "fp32":
            clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        env.simulate(DT, K, bfb.STEP_DIFFUSION)
        e1.record(stream)
        e1.synchronize()
        ms = slowest(e0.elapsed_time(e1))
        clk = clocks.stop() if name == "fp32" else None
        barrier()
        # per-kernel device time (events around every launch, same stream)
        prof = env.profile_steps(DT, min(K, 50), bfb.STEP_DIFFUSION)
        nprof = min(K, 50)
        results[name] = dict(ms=ms, clocks=clk, prof=prof, nprof=nprof, env=env, elem=4 if prec == bfb.FP32 else 8,
                             tuning=tuned)

    # both envs ran the same steps from the same field: FP32's error against FP64
    n_steps_run = warm + K + min(K, 50)
    err_linf, err_l2 = results["fp32"]["env"].compare(results["fp64"]["env"])
    results["fp64"]["env"].close()

    # end to end through the C ABI with reference-facing host buffers
    env = results["fp32"]["env"]
    host = torch.from_numpy(rho0.reshape(-1).copy()).pin_memory()
    K_e2e = max(1, min(K, 20))
    env.step_host_ptr(host.data_ptr(), DT, 1)  # warm
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K_e2e):
        env.step_host_ptr(host.data_ptr(), DT, 1)
    e1.record(stream)
    e1.synchronize()
    ms_e2e = slowest(e0.elapsed_time(e1))

    # reverse mode on the same FP32 env: n_adj steps, with and without segment recompute
    n_adj = 20
    w = torch.randn(V * S, device=f"cuda:{local}", dtype=torch.float32)
    adj_ms = {}
    for Kc in (n_adj, 5):
        env.set_field(rho0)
        torch.cuda.synchronize()
        env.adjoint_run(DT, n_adj, w.data_ptr(), checkpoint_every=Kc)  # warm: workspace
        env.set_field(rho0)
        barrier()
        e0.record(stream)
        env.adjoint_run(DT, n_adj, w.data_ptr(), checkpoint_every=Kc)
        e1.record(stream)
        e1.synchronize()
        adj_ms[Kc] = slowest(e0.elapsed_time(e1))
    # the same run when only dL/du0 is wanted: no D / lambda gradients, no per-line sums
    env.set_field(rho0)
    barrier()
    e0.record(stream)
    env.adjoint_run(DT, n_adj, w.data_ptr(), checkpoint_every=n_adj, coef_grads=False)
    e1.record(stream)
    e1.synchronize()
    adj_field_ms = slowest(e0.elapsed_time(e1))
    env.close()

    # the uneven ensemble at N = 1: batched launches against the per-instance loop
    ens = None
    if world == 1 and not args.no_ensemble:
        specs = ensemble_specs()
        envs = [build_instance(bfb, sp, bfb.FP32, local) for sp in specs]
        K_ens = max(1, min(K, 20))
        t = time_ensemble(bfb, envs, K_ens, stream)
        vs = sum(int(np.prod(sp["shape"])) * sp["S"] for sp in specs)
        step_bytes_ens = 6.0 * vs * 4
        for e in envs:
            e.close()
        peak_e, _ = measured_peak()
        ens = {"workload": f"{len(specs)} independent microenvironments, edges U{{32..160}} per axis, 1-6 "
                           "substrates, 0-20k agents each, x-face Dirichlet on substrate 0, FP32, diffusion + agents",
               "voxel_substrates": vs, "steps": K_ens,
               "batch_ms_per_step": t["batch"], "loop_ms_per_step": t["loop"],
               "batch_autotuned": t["tuned"], "mode_ms_per_step": t["modes"],
               "batch_value": vs / (t["batch"] / 1e3), "loop_value": vs / (t["loop"] / 1e3),
               "batch_over_loop_time": t["batch"] / t["loop"],
               "step_roofline_frac": {"batch": step_bytes_ens / (t["batch"] / 1e3) / 1e9 / peak_e,
                                      "loop": step_bytes_ens / (t["loop"] / 1e3) / 1e9 / peak_e},
               "note": "step roofline counts 6 V*S*4 bytes per step (three sweeps); CUDA events on one stream"}

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    r32, r64 = results["fp32"], results["fp64"]
    value = world * V * S * K / (r32["ms"] / 1e3)
    value64 = world * V * S * K / (r64["ms"] / 1e3)
    peak, peak_src = measured_peak()
    phases = ["sweep_x", "sweep_y", "sweep_z"]
    per = r32["prof"][:3] / r32["nprof"]  # ms per launch
    dom = int(np.argmax(per))
    bytes_launch = 2.0 * V * S * 4  # one read + one write of the field
    achieved = bytes_launch / (per[dom] / 1e3) / 1e9
    step_bytes = 6.0 * V * S * 4
    ms_step = r32["ms"] / K
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        r = cpu_reference_run(args.cpu_seconds, min_steps=1)
        if r is not None:
            rate, n, threads, sname, el = r
            cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference", "cpu": cpu_model(),
                   "sample": f"{n} full {NX}^3x{S} FP64 steps ({el:.1f} s) of the reference {sname} "
                             "(faster of LOD_3D / AVX256D), after one factor-setup step"}
        else:
            rate, n = cpu_port_run(args.cpu_seconds)
            cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port", "cpu": cpu_model(),
                   "sample": f"{n} steps of a 64^3x8 sample with the oracle port (reference not built)"}
    line = {
        "metric": metric_name(), "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": warm,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded U[0,1) field, log-uniform D/lambda)",
        "config": config(),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": ncu_traffic(f"fp32_{phases[dom]}") if (NX, S) == (256, 8) else None,
                     "kernel": phases[dom],
                     "algorithmic_bytes_per_launch": bytes_launch, "peak_source": peak_src,
                     "ms_per_launch": float(per[dom])},
        "step_roofline": {"achieved": step_bytes / (ms_step / 1e3) / 1e9, "frac": step_bytes / (ms_step / 1e3) / 1e9 / peak,
                          "algorithmic_bytes_per_step": step_bytes},
        "kernel_ms_per_launch": {p: float(x) for p, x in zip(phases, per)},
        "fp64": {"value": value64, "ms_per_step": r64["ms"] / K,
                 "step_roofline_frac": 6.0 * V * S * 8 / (r64["ms"] / K / 1e3) / 1e9 / peak,
                 "kernel_ms_per_launch": {p: float(x) for p, x in zip(phases, r64["prof"][:3] / r64["nprof"])}},
        "fp32_over_fp64": value / value64,
        "tuning": {"fp32": r32["tuning"], "fp64": r64["tuning"],
                   "fields": "per sweep x, y, z: (TMA tiles 1 / cp.async 0, warps per CTA, row groups per tile), "
                             + ("the library defaults" if args.no_autotune else "chosen by bfb_autotune before the warm-up")},
        "fp32_error_vs_fp64": {"rel_linf": err_linf, "rel_l2": err_l2, "after_steps": n_steps_run},
        "clocks": r32["clocks"],
        "e2e": {"value": world * V * S * K_e2e / (ms_e2e / 1e3), "unit": UNIT, "h2d_bytes_per_step": V * S * 8,
                "d2h_bytes_per_step": V * S * 8, "steps": K_e2e,
                "path": "bfb_step_host: pinned FP64 host field -> device (FP32) -> 1 LOD step -> host"},
        "gpu_launches": 3 * K,
        "cpu_baseline": cpu,
        "adjoint": {
            "workload": f"bfb_adjoint_run, FP32 {NX}^3x{S}, {n_adj} steps, dL/du_final random",
            "forward_ms_per_step": ms_step,
            "run_ms_per_step": {f"checkpoint_every_{k}": v / n_adj for k, v in adj_ms.items()},
            # the run = forward (writing the last segment's stage fields) + recompute of earlier segments + reverse
            "reverse_ms_per_step": adj_ms[n_adj] / n_adj - ms_step,
            "reverse_over_forward": (adj_ms[n_adj] / n_adj - ms_step) / ms_step,
            "run_over_forward": {f"checkpoint_every_{k}": v / n_adj / ms_step for k, v in adj_ms.items()},
            "without_D_lambda_gradients": {
                "run_ms_per_step": adj_field_ms / n_adj,
                "reverse_over_forward": (adj_field_ms / n_adj - ms_step) / ms_step,
                "run_over_forward": adj_field_ms / n_adj / ms_step},
        },
        "ensemble": ens,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ensemble_arm(args):
    """The uneven ensemble sharded across ranks: each rank steps its share of
    the instances (greedy bytes balancing, ranks.local_instances) as one
    batch; no collective touches the fields. value = all ranks' voxel*substrate
    updates per step / the slowest rank's step time. Per-instance checksums
    are gathered by instance at the end."""
    import torch
    rank, world, local = dist_setup(args)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    bfb = load_bfb()
    ranks = importlib.import_module("biofvm_b_b200.ranks")
    specs = ensemble_specs()
    weights = [ranks.instance_bytes(sp["shape"], sp["S"], 4) for sp in specs]
    mine = ranks.local_instances(weights, rank, world)
    envs = [build_instance(bfb, specs[i], bfb.FP32, local) for i in mine]
    vs_all = sum(int(np.prod(sp["shape"])) * sp["S"] for sp in specs)
    vs_mine = sum(int(np.prod(specs[i]["shape"])) * specs[i]["S"] for i in mine)
    flags = bfb.STEP_DIFFUSION | bfb.STEP_CELLS
    warm, K = max(args.warmup, 3), args.steps
    stream = torch.cuda.Stream(device=dev)
    batch = bfb.Batch(envs)
    batch.set_stream(stream.cuda_stream)
    tuned, _ = batch.autotune(DT, flags, trials=2)  # mode and launch shape; the fields are restored
    tuned = {"mode": BATCH_MODE_NAMES[batch.mode], "warps_per_cta": tuned[0], "tiles_per_item": tuned[1]}
    batch.simulate(DT, warm, flags)
    stream.synchronize()
    rank_barrier(dev)
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.simulate(DT, K, flags)
    e1.record(stream)
    e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dev)
    clk = clocks.stop()
    batch.synchronize()
    rank_barrier(dev)
    # end to end: every step uploads each local instance's field from pinned
    # host memory, steps the batch, and reads every field back
    for e in envs:
        e.set_stream(stream.cuda_stream)
    hosts = [torch.empty(int(np.prod(specs[i]["shape"])) * specs[i]["S"], dtype=torch.float32).pin_memory()
             for i in mine]
    def raw(call, e, h):
        if call(e.h, ctypes.c_void_p(h.data_ptr())) != 0:
            raise RuntimeError(e.L.bfb_last_error().decode())

    for h, e in zip(hosts, envs):
        raw(e.L.bfb_get_field_raw, e, h)
    K_e2e = max(1, min(K, 5))
    rank_barrier(dev)
    e0.record(stream)
    for _ in range(K_e2e):
        for h, e in zip(hosts, envs):
            raw(e.L.bfb_set_field_raw, e, h)
        batch.simulate(DT, 1, flags)
        for h, e in zip(hosts, envs):
            raw(e.L.bfb_get_field_raw, e, h)
    e1.record(stream)
    e1.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), dev)
    sums = gather_by_instance(mine, [e.checksum() for e in envs], len(specs), 6, dev)
    batch.close()
    for e in envs:
        e.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    peak, _ = measured_peak()
    step_bytes = 6.0 * vs_all * 4
    line = {
        "metric": f"voxel*substrate updates/s per LOD step (uneven ensemble, {len(specs)} instances)",
        "value": vs_all / (ms / K / 1e3), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": warm,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded per instance: U[0,1) fields, log-uniform D/lambda and agent rates)",
        "config": {"workload": f"{len(specs)} independent microenvironments, edges U{{32..160}} per axis, 1-6 "
                               "substrates, 0-20k agents each, x-face Dirichlet 38 on substrate 0, diffusion + agents",
                   "voxel_substrates": vs_all, "l2": "inputs larger than L2 (3.2 GB of FP32 fields)",
                   "parallelism": f"instances sharded over {world} rank(s) by greedy bytes balancing, one batch per rank"},
        "roofline": {"bound": "hbm", "achieved": step_bytes / (ms / K / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": step_bytes / (ms / K / 1e3) / 1e9 / peak, "traffic": None,
                     "kernel": "whole step (three sweeps of every instance)"},
        "clocks": clk,
        "e2e": {"value": vs_all * K_e2e / (ms_e2e / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": vs_all * 4, "d2h_bytes_per_step": vs_all * 4, "steps": K_e2e,
                "path": "bfb_set_field_raw per instance (pinned FP32) -> bfb_batch_simulate -> bfb_get_field_raw"},
        "gpu_launches": None,
        "checksum_of_checksums": float(sums.sum()),
        "rank0_share": vs_mine / vs_all,
        "batch_autotuned": tuned,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_slabs_arm(args):
    """One FP64 grid split into x slabs over the ranks (the reference's MPI
    decomposition, BioFVM_parallel.cpp:108-144): each rank holds one slab
    env, the x lines are solved with the pipelined exchange of boundary
    planes (slabs.step; NCCL send/recv between neighbouring ranks), the y and
    z sweeps are local. value = the grid's voxel*substrate updates per step /
    the slowest rank's step time."""
    import torch
    rank, world, local = dist_setup(args)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    bfb = load_bfb()
    slabs = importlib.import_module("biofvm_b_b200.slabs")
    x0, m = slabs.split_planes(NX, world)[rank]
    D, lam, _ = coefficients()
    field = np.random.default_rng(SEED + 1 + rank).random((m, NY, NZ, S))
    slab = bfb.SlabEnv(NX, x0, m, NY, NZ, S, dx=DX, device=local)
    slab.set_coefficients(D, lam)
    slab.set_field(field)
    stream = torch.cuda.Stream(device=dev)
    slab.set_stream(stream.cuda_stream)
    planes = {k: torch.zeros(slab.lines, dtype=torch.float64, device=dev) for k in slabs.PLANES}

    class Planes:
        def ptr(self, name):
            return planes[name].data_ptr()

    class Nccl:  # point-to-point messages on the slab's stream
        def send(self, name, l0, l1, peer):
            dist.send(planes[name][l0:l1], dst=peer)

        def recv(self, name, l0, l1, peer):
            dist.recv(planes[name][l0:l1], src=peer)

    blocks = 8 if world > 1 else 1  # blocks only pipeline the ranks
    warm, K = max(args.warmup, 3), max(1, min(args.steps, 200))
    with torch.cuda.stream(stream):
        for _ in range(warm):
            slabs.step(slab, DT, rank, world, Planes(), Nccl(), blocks)
        stream.synchronize()
        rank_barrier(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            slabs.step(slab, DT, rank, world, Planes(), Nccl(), blocks)
        e1.record(stream)
        e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dev)
    total = sum_over_ranks(float(np.sum(slab.checksum())), dev)
    slab.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    vs = NX * NY * NZ * S
    line = {
        "metric": f"voxel*substrate updates/s per LOD step ({NX}^3 voxels x {S} substrates, x slabs)",
        "value": vs / (ms / K / 1e3), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": warm,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded U[0,1) field per slab, log-uniform D/lambda)",
        "config": {"workload": f"LOD diffusion-decay step, {NX}^3 voxels x {S} substrates, dt={DT}, dx={DX}, "
                               f"split into {world} x slab(s)",
                   "l2": "inputs larger than L2", "parallelism": f"x slabs over {world} rank(s), {blocks} line blocks"},
        "gpu_launches": None,
        "checksum_of_checksums": total,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-seconds", type=float, default=60.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", type=int, default=256, help="edge of the cubic grid (profiling small cases)")
    ap.add_argument("--substrates", type=int, default=8)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shapes (for profiler runs, whose timing would mislead the tuner)")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the uneven-ensemble block of the default run")
    ap.add_argument("--workload", default="grid", choices=["grid", "ensemble", "slabs"],
                    help="grid: the 256^3 x 8 step (replicas per GPU); ensemble: 256 uneven instances sharded over "
                         "the GPUs; slabs: one FP64 grid split into x slabs over the GPUs")
    args = ap.parse_args()
    global NX, NY, NZ, S
    NX = NY = NZ = args.grid
    S = args.substrates
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "ensemble":
        return run_ensemble_arm(args)
    if args.workload == "slabs":
        return run_slabs_arm(args)
    return run_our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
