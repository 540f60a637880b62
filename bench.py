#!/usr/bin/env python
"""Benchmark of the per-step microenvironment update on B200 GPUs.

One step is the reference driver's loop body (paraBioFVM src/main.cpp:68-107): LOD diffusion
(x, y, z Thomas sweeps with the Dirichlet overwrites), the central-difference gradient, and
secretion/uptake, with the agent binning rebuilt every 10th step.  The default workload is the
large plain configuration: a 320 x 320 x 320 mesh (dx = 20 um), 16 FP32 substrates, 1,000,000 agents
in 32 Gaussian clusters, Dirichlet 1.0 for substrate 0 on every face and 1 % of the interior voxels
pinned to U(0,1) values; all data seeded and synthetic.

Reported: ``value`` = voxel*substrate updates per second over all GPUs, device-timed with CUDA
events on the solver's stream over ``--steps`` graph-replayed steps (inputs stay resident; the 2.1
GB field is far larger than L2, so no flush is needed); ``e2e`` = the same metric through the C ABI
with pinned host buffers (state stored, steps called one solver at a time, field, gradients and
internalized substrates loaded back, all inside the timed region); ``roofline`` of the dominant
kernel; ``cpu_baseline`` = the CPU oracle on the host cores.  ``--impl reference`` times the CPU
restatement of the reference's host solvers (the reference itself cannot be built in this image).

``--workload batch-256`` measures the batched-ensemble form instead: 256 independent meshes (edge
U{24..96} voxels, 1..8 substrates, 100..20,000 agents, per-instance coefficients) stepped together
as one CUDA graph (bfvm_batch_run_steps), against the same instances stepped one after another on
one stream.

Multi-GPU: the plain single-mesh step does not shard (its z sweep couples the whole mesh), so
``--gpus N`` runs N independent replicas, one per GPU (weak scaling, no collective on the data
path); the device time is the maximum over ranks.

``--workload zslab-320`` splits the plain-320 mesh along z instead (parabiofvm_b200.slabs): under
torchrun one slab per rank, joined by an NCCL all-gather of the z sweep's line carries and a
neighbour exchange of edge planes (strong scaling: one mesh over all ranks); in a single process
``--slabs K`` slabs on one GPU joined by copies, which measures what the split itself costs against
the same mesh in one solver.
"""

from __future__ import annotations

import argparse
import json
import os
import signal
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOADS = {
    # the large plain configuration (headline)
    "plain-320": dict(edge=320, S=16, agents=1_000_000, clustered=True, sigma=200.0, interior_fraction=0.01,
                      seed=20261203,
                      text="320^3 voxels (dx 20 um) x 16 FP32 substrates, 1,000,000 agents in 32 Gaussian clusters "
                           "(sigma 200 um), 1% interior Dirichlet voxels, Dirichlet 1.0 on substrate 0 at all faces, "
                           "dt 0.01 min, binning rebuilt every 10th step"),
    # the large configuration at half the edge, for ncu captures (262 MB field, still larger than L2)
    "plain-160": dict(edge=160, S=16, agents=125_000, clustered=True, sigma=200.0, interior_fraction=0.01,
                      seed=20261203,
                      text="160^3 voxels (dx 20 um) x 16 FP32 substrates, 125,000 agents in 32 Gaussian clusters, "
                           "1% interior Dirichlet voxels, Dirichlet 1.0 on substrate 0 at all faces (profiling size)"),
    # the CPU-runnable configuration (parity case, L2-resident)
    "plain-50": dict(edge=50, S=4, agents=5000, clustered=False, sigma=0.0, interior_fraction=0.0, seed=11,
                     text="50^3 voxels x 4 FP32 substrates, 5,000 uniform agents, Dirichlet 1.0 on substrate 0 at "
                          "all faces, dt 0.01 min"),
}

METRIC = "voxel·substrate steps/s, % HBM peak; speedup vs plain GPU at ≤1e-3 rel L2"
UNIT = "voxel*substrate updates/s"
FALLBACK_HBM_GBS = 6650.0


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_workload(name, seed_offset=0):
    from parabiofvm_b200.workloads import synthetic

    w = WORKLOADS[name]
    return synthetic(w["edge"], w["S"], w["agents"], w["seed"] + seed_offset, clustered=w["clustered"],
                     sigma=w["sigma"] or 200.0, interior_fraction=w["interior_fraction"])


def algorithmic_step_bytes(w, recompute_fraction=0.1):
    """Bytes a step must move at minimum: 3 sweeps x (read + write) + gradient written, 4 B each
    per voxel*substrate (36 B), plus the agent terms (per-voxel reductions read, density
    read-modify-write, internalized intermediates and read-modify-write) and the Dirichlet data."""
    VS = w.voxel_count * w.S
    A = w.agents.count if w.agents is not None else 0
    n_d = 0 if w.interior_voxels is None else len(w.interior_voxels)
    agent = A * w.S * (20 + (20 if w.compute_internalized else 0)) + 16 * A
    recompute = recompute_fraction * A * w.S * (16 + 24)
    return 36 * VS + agent + recompute + 5 * n_d * w.S


def dirichlet_elements(w):
    """Conditioned elements of the workload: face voxels with a condition (each voxel once) and
    interior voxels with a condition (the bound the overwrite list stays within)."""
    n = 0
    ext = list(w.grid) + [1] * (3 - len(w.grid))
    for (dim, is_max), (vals, conds) in w.boundary.items():
        others = [ext[d] for d in range(3) if d != dim]
        n += int(np.count_nonzero(conds)) * others[0] * others[1]
    if w.interior_conditions is not None:
        n += int(np.count_nonzero(w.interior_conditions))
    return n


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def committed_traffic():
    """Per-launch DRAM bytes of each kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return {}


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"bfvm_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "50"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.send_signal(signal.SIGTERM)
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [t.strip() for t in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max((float(r[3]) for r in rows if r[3].replace(".", "").isdigit()), default=None)}


def physical_gpu_index(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [t.strip() for t in vis.split(",") if t.strip()]
        if local_rank < len(ids):
            return ids[local_rank]
    return str(local_rank)


def make_oracle_for(w, dtype):
    import oracle

    oracle.build()
    oracle.set_threads(os.cpu_count() or 1)
    o = oracle.Oracle(w.dims, w.bbox_min, w.bbox_max, w.voxel_shape, w.diffusion_coefficients, w.decay_rates,
                      w.time_step, w.initial_conditions, w.compute_internalized, dtype=dtype)
    for (dim, is_max), (vals, conds) in w.boundary.items():
        o.set_boundary_dirichlet(dim, is_max, vals, conds)
    if w.interior_voxels is not None:
        o.set_interior_dirichlet(w.interior_voxels, w.interior_values, w.interior_conditions)
    o.set_densities(w.densities)
    if w.agents is not None:
        a = w.agents
        o.set_agents(a.secretion_rates, a.saturation_densities, a.uptake_rates, a.net_export_rates, a.internalized,
                     a.fraction_released, a.volumes, a.positions)
    o.initialize()
    return o


def _max_rel(a, r):
    a = np.asarray(a, np.float64).reshape(-1)
    r = np.asarray(r, np.float64).reshape(-1)
    floor = max(float(np.abs(r).max()) * 1e-6, 1e-30)
    return float((np.abs(a - r) / np.maximum(np.abs(r), floor)).max())


def _rel_l2(a, r):
    a = np.asarray(a, np.float64).reshape(-1)
    r = np.asarray(r, np.float64).reshape(-1)
    return float(np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-300))


def parity_report(workload, steps, with_fp64):
    """The GPU step against the oracle (FP32, and FP64 when asked) after `steps` full steps of the
    workload from its initial state: max relative error (floor 1e-6 of max|ref|) and rel-L2."""
    from parabiofvm_b200.workloads import make_solver

    w = make_workload(workload)
    g = make_solver(w)
    g.run_steps(steps, 0)
    g.synchronize()
    got = g.load_densities().copy()
    g.close()
    out = {"workload": workload, "steps": steps}
    for name, dt in (("fp32", np.float32),) + ((("fp64", np.float64),) if with_fp64 else ()):
        o = make_oracle_for(w, dt)
        o.run_steps(steps, 0)
        ref = o.densities()
        o.close()
        out[f"max_rel_vs_{name}"] = _max_rel(got, ref)
        out[f"rel_l2_vs_{name}"] = _rel_l2(got, ref)
        if name == "fp64":
            # the FP32 reference algorithm's own distance to the FP64 one, for scale
            o32 = make_oracle_for(w, np.float32)
            o32.run_steps(steps, 0)
            out["rel_l2_fp32_oracle_vs_fp64"] = _rel_l2(o32.densities(), ref)
            o32.close()
    return out


def step_parity(workload, steps):
    """The GPU against the FP32 and FP64 oracles, all three stepping in lockstep from the same
    initial state (recompute every 10th step), compared after steps 1, 2, 5, 10, 20, 50, 100 (those
    up to `steps`, and `steps`): maximum relative error (floor 1e-6 of max|ref|) and rel-L2 of the
    densities."""
    from parabiofvm_b200.workloads import make_solver

    w = make_workload(workload)
    g = make_solver(w)
    o32 = make_oracle_for(w, np.float32)
    o64 = make_oracle_for(w, np.float64)
    checks = sorted({k for k in (1, 2, 5, 10, 20, 50, 100) if k <= steps} | {steps})
    rows = []
    t0 = time.perf_counter()
    for k in range(steps):
        g.run_steps(1, k)
        o32.run_steps(1, k)
        o64.run_steps(1, k)
        if k + 1 not in checks:
            continue
        got = g.load_densities()
        r32, r64 = o32.densities(), o64.densities()
        rows.append({"step": k + 1, "max_rel_vs_fp32": _max_rel(got, r32), "rel_l2_vs_fp32": _rel_l2(got, r32),
                     "max_rel_vs_fp64": _max_rel(got, r64), "rel_l2_vs_fp64": _rel_l2(got, r64),
                     "rel_l2_fp32_oracle_vs_fp64": _rel_l2(r32, r64)})
        log(f"step {k + 1}: max rel vs fp32 {rows[-1]['max_rel_vs_fp32']:.3e}, "
            f"vs fp64 {rows[-1]['max_rel_vs_fp64']:.3e} ({time.perf_counter() - t0:.0f}s)")
    g.close()
    o32.close()
    o64.close()
    return {"workload": workload, "steps": steps, "checks": rows}


def host_cpu_model():
    """The host CPU's model name (the first 'model name' of /proc/cpuinfo), or None."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_oracle_rate(w, budget_s=20.0, max_steps=3):
    """Time the CPU oracle (all host threads) on the workload: voxel*substrate updates/s."""
    import oracle

    oracle.build()
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    from oracle import Oracle

    o = Oracle(w.dims, w.bbox_min, w.bbox_max, w.voxel_shape, w.diffusion_coefficients, w.decay_rates, w.time_step,
               w.initial_conditions, w.compute_internalized, dtype=np.float32)
    for (dim, is_max), (vals, conds) in w.boundary.items():
        o.set_boundary_dirichlet(dim, is_max, vals, conds)
    if w.interior_voxels is not None:
        o.set_interior_dirichlet(w.interior_voxels, w.interior_values, w.interior_conditions)
    o.set_densities(w.densities)
    a = w.agents
    o.set_agents(a.secretion_rates, a.saturation_densities, a.uptake_rates, a.net_export_rates, a.internalized,
                 a.fraction_released, a.volumes, a.positions)
    o.initialize()
    times = []
    total = 0.0
    step = 0
    while step < max_steps and (total < budget_s or step == 0):
        t0 = time.perf_counter()
        o.run_steps(1, step)
        dt = time.perf_counter() - t0
        times.append(dt)
        total += dt
        step += 1
    o.close()
    VS = w.voxel_count * w.S
    return VS * len(times) / total, threads, times


def run_reference_batch(args, threads):
    """The reference arm of batch-256: the reference steps one mesh at a time, so the CPU port steps
    the instances one after another, as many as fit the time budget (one warm-up step each)."""
    ws = make_batch()
    budget = args.reference_budget_s
    units = 0
    elapsed = 0.0
    done = 0
    for w in ws:
        o = make_oracle_for(w, np.float32)
        o.run_steps(1, 1)
        t0 = time.perf_counter()
        o.run_steps(1, 2)
        elapsed += time.perf_counter() - t0
        units += w.voxel_count * w.S
        done += 1
        o.close()
        if elapsed > budget:
            break
    value = units / elapsed
    sample = f"one step of each of the first {done} of {len(ws)} instances, one after another (budget {budget:.0f}s)"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": int(args.gpus),
        "steps": 1, "warmup": 1, "ms_per_step": 1e3 * elapsed * len(ws) / done, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": "batch-256: 256 independent meshes, edge U{24..96}, 1..8 substrates, 100..20,000 "
                               "clustered agents, per-instance coefficients",
                   "implementation": "CPU restatement of src/solver/host (OpenMP, -O3, no FP contraction)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "cpu_model": host_cpu_model(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's host step on all host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle

    oracle.build()
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    if args.workload == "batch-256":
        return run_reference_batch(args, threads)
    if args.workload == "surrogate-128":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned surrogate; its CPU step "
                                                              "is timed by the plain workloads' reference arm"}),
              flush=True)
        return 0
    # the reference holds a mesh in one solver: a split mesh is timed whole
    name = "plain-320" if args.workload == "zslab-320" else args.workload
    t_setup = time.perf_counter()
    w = make_workload(name)
    log(f"reference arm: workload built in {time.perf_counter() - t_setup:.1f}s")
    o = make_oracle_for(w, np.float32)
    # warm-up steps, then as many timed steps of --steps as fit in the time budget
    t_step = None
    for i in range(args.warmup):
        t0 = time.perf_counter()
        o.run_steps(1, i)
        t_step = time.perf_counter() - t0
    budget = args.reference_budget_s
    timed = args.steps if t_step is None else max(1, min(args.steps, int(budget // max(t_step, 1e-9))))
    t0 = time.perf_counter()
    o.run_steps(timed, args.warmup)
    elapsed = time.perf_counter() - t0
    VS = w.voxel_count * w.S
    value = VS * timed / elapsed
    sample = (f"{timed} of {args.steps} requested full steps of the workload after {args.warmup} warm-up steps "
              f"(time budget {budget:.0f}s)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": int(args.gpus),
        "steps": timed, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / timed, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"{args.workload}: {WORKLOADS[name]['text']}",
                   "implementation": "CPU restatement of src/solver/host (OpenMP, -O3, no FP contraction)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "cpu_model": host_cpu_model(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


BATCH_INSTANCES = 256


BATCH_TEXT = ("256 independent meshes, edge U{24..96}, 1..8 substrates, 100..20,000 clustered agents, "
              "per-instance coefficients, recompute every 10th step")


def make_batch(seed=20261204, count=BATCH_INSTANCES):
    """The ensemble of the batch-256 workload: per instance a cubic mesh of edge U{24..96},
    U{1..8} substrates and U{100..20000} clustered agents, each with its own coefficients."""
    from parabiofvm_b200.workloads import synthetic

    rng = np.random.default_rng(seed)
    ws = []
    for i in range(count):
        edge = int(rng.integers(24, 97))
        S = int(rng.integers(1, 9))
        A = int(rng.integers(100, 20001))
        ws.append(synthetic(edge, S, A, seed + 1 + i, clustered=True, sigma=100.0, interior_fraction=0.0))
    return ws


def measure_batch(steps, warmup, clocks=True):
    """The batched-ensemble workload on one GPU.  Two copies of every instance are made: one set is
    stepped as a batch (one graph per step), the other one instance after another on one stream
    (bfvm_run_steps), over the same steps from the same state.  Returns the two device times, the
    launches of the batched steps and the largest relative L2 distance between an instance's two
    fields."""
    import torch

    from parabiofvm_b200 import Batch
    from parabiofvm_b200.workloads import make_solver

    t_setup = time.perf_counter()
    ws = make_batch()
    units = sum(w.voxel_count * w.S for w in ws)
    log(f"batch: {len(ws)} instances, {units / 1e6:.1f} M voxel*substrates, built in "
        f"{time.perf_counter() - t_setup:.1f}s")
    stream = torch.cuda.Stream()
    batched = [make_solver(w) for w in ws]
    alone = [make_solver(w) for w in ws]

    def timed(run):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    for s in batched + alone:
        s.set_stream(stream.cuda_stream)
    b = Batch(batched)
    tuned = b.autotune()
    b.run_steps(warmup, 0)
    b.synchronize()
    sampler = ClockSampler(physical_gpu_index(0)) if clocks else None
    if sampler:
        sampler.start()
        time.sleep(1.0)
    launches0 = sum(s.launch_count for s in batched)
    ms_batch = timed(lambda: b.run_steps(steps, warmup))
    launches = sum(s.launch_count for s in batched) - launches0
    clock_rec = sampler.stop() if sampler else None
    b.close()

    # one instance after another: the same warm-up steps untimed, then the same steps timed
    for k in range(warmup):
        for s in alone:
            s.run_steps(1, k)

    def sequential():
        for k in range(steps):
            for s in alone:
                s.run_steps(1, warmup + k)

    ms_seq = timed(sequential)
    worst = 0.0
    for sb, sa in zip(batched, alone):
        worst = max(worst, _rel_l2(sb.load_densities(), sa.load_densities()))
    for s in batched + alone:
        s.close()
    return {"instances": len(ws), "voxel_substrates": units, "ms_batch": ms_batch, "ms_sequential": ms_seq,
            "launches": launches, "clocks": clock_rec, "max_rel_l2_vs_alone": worst, "autotuned": tuned}


def run_batch(args):
    """The batched-ensemble workload on one GPU: batched (one graph) and sequential (one stream)."""
    r = measure_batch(args.steps, args.warmup)
    units = r["voxel_substrates"]
    value = units * args.steps / (r["ms_batch"] / 1e3)
    seq = units * args.steps / (r["ms_sequential"] / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["ms_batch"] / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"batch-256: {BATCH_TEXT}", "instances": r["instances"], "voxel_substrates": units,
                   "l2": "ensemble fields 4x the L2, no flush"},
        "sequential": {"value": seq, "ms_per_step": r["ms_sequential"] / args.steps,
                       "what": "the same instances stepped one after another on one stream (bfvm_run_steps)"},
        "speedup_vs_sequential": value / seq,
        "max_rel_l2_vs_alone": r["max_rel_l2_vs_alone"],
        "autotuned": r["autotuned"],
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
    }
    print(json.dumps(line), flush=True)
    return 0


def reduce_max_over_ranks(x, world, device):
    """The largest of every rank's ``x`` (the job's time is its slowest replica's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, steps, ms):
    """Units every rank processed over the slowest rank's time: replicas do equal work."""
    return world * units_per_rank * steps / (ms / 1e3)


def measured_tensor_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured (cuBLAS bf16, burst)"
    except Exception:
        return 1590.0, "fallback"


SURROGATE_TEXT = ("128^3 voxels (dx 20 um) x 4 FP32 substrates; network: 3x3x3 conv to 32 channels, 4 residual "
                  "blocks of two 3x3x3 convs, 3x3x3 projection, bf16 weights and activations, f32 accumulate; "
                  "training pairs from the plain GPU solver (fields of 8 Gaussian bumps, 10k-100k uniform agents, "
                  "16 steps), Adam lr 1e-3 batch 4; inference with 200,000 clustered agents, 100 macro-steps of 16 "
                  "steps, every 8th re-run plain, plain takes over above 1e-3 relative L2")


def measure_surrogate(train_steps=10, warmup=3, fallback_macro_steps=100, fresh_train_steps=0):
    """The learned surrogate at 128^3 x 4.

    - Training throughput: Adam steps at batch 4 on one batch of pairs from the plain solver
      (device-timed, no loss read-back), on a network of its own.
    - One forward convolution at batch 4 against the tensor peak (the roofline numerator).
    - One macro-step of the trained network (the committed parameters, trained by
      parabiofvm_b200.surrogate_train) against 16 plain steps with 200,000 clustered agents.
    - The fallback controller over 1,600 steps with the trained network, against plain stepping.
    Without committed parameters the controller's network gets `fresh_train_steps` Adam steps on
    fresh pairs instead."""
    import ctypes

    import torch

    from parabiofvm_b200 import _abi
    from parabiofvm_b200 import surrogate as su

    torch.cuda.set_device(0)
    env = su.standard_environment()
    S = env.S
    B = 4
    net = su.Surrogate(env.grid, S, max_batch=B, seed=7)
    gen = su.PairGenerator(env, seed=11)
    VS = env.voxels * S
    with torch.cuda.stream(net.stream):
        field, src, sink, target, pred = [torch.empty((B, VS), device="cuda") for _ in range(5)]

    def events():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    # pairs from the plain solver
    t0 = time.perf_counter()
    gen.batch(field, src, sink, target)
    torch.cuda.synchronize()
    pair_s = (time.perf_counter() - t0) / B

    # training steps on that batch (device-timed; no loss read-back inside the timed region)
    net.stream.wait_stream(gen.stream)
    for _ in range(warmup):
        net.train_step(field, src, sink, target, pred, 1e-3, read_loss=False)
    net.synchronize()
    e0, e1 = events()
    e0.record(net.stream)
    for _ in range(train_steps):
        net.train_step(field, src, sink, target, pred, 1e-3, read_loss=False)
    e1.record(net.stream)
    net.synchronize()
    ms_train = e0.elapsed_time(e1) / train_steps
    conv_flop = 2.0 * 27 * 32 * 32 * env.voxels * B
    train_flop = conv_flop * (10 + 9 + 10)  # forward, input gradients (not of layer 0), weight gradients

    # the network the controller runs: the committed trained parameters, else a short training
    run_net = su.Surrogate(env.grid, S, max_batch=1, seed=7, stream=net.stream)
    trained = None
    if os.path.exists(su.WEIGHTS_PATH):
        rec = su.load_trained(run_net, env)
        trained = {"parameters": os.path.relpath(su.WEIGHTS_PATH, ROOT), "best_epoch": rec["best_epoch"],
                   "training_steps": rec["best_epoch"] * (rec["recipe"]["pairs"] // rec["recipe"]["batch"]),
                   "pairs": rec["recipe"]["pairs"], "held_out_rel_l2": rec["held_out_rel_l2"],
                   "held_out_rel_l2_without_net": rec["held_out_rel_l2_without_net"]}
    else:
        losses = su.train(run_net, gen, steps=fresh_train_steps, batch=1, learning_rate=1e-3)
        trained = {"parameters": None, "training_steps": len(losses)}

    # one forward convolution at batch 4: the roofline numerator
    lib = _abi.load()
    xin = torch.randn((B, env.voxels, 32), device="cuda").to(torch.bfloat16)
    w = (torch.randn((27, 32, 32), device="cuda") * 0.05).to(torch.bfloat16)
    yout = torch.empty_like(xin)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    shape = (ctypes.c_int32 * 4)(*env.grid, B)
    stream = torch.cuda.current_stream()

    def conv_once():
        _abi.check(lib.bfvm_sur_conv3d(shape, ctypes.c_void_p(xin.data_ptr()), ctypes.c_void_p(w.data_ptr()), None, None,
                                       0, None, ctypes.c_void_p(yout.data_ptr()), None, None, 0,
                                       ctypes.c_void_p(err.data_ptr()), ctypes.c_void_p(stream.cuda_stream)))

    for _ in range(3):
        conv_once()
    torch.cuda.synchronize()
    reps = 10
    e0, e1 = events()
    e0.record(stream)
    for _ in range(reps):
        conv_once()
    e1.record(stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ms_conv = e0.elapsed_time(e1) / reps
    del xin, w, yout
    peak, peak_kind = measured_tensor_peak()
    achieved = conv_flop / (ms_conv / 1e3) / 1e12

    # a macro-step of the network against 16 plain steps, 200,000 clustered agents
    agents = su.random_agents(env, np.random.default_rng(13), 200_000, clustered=True)
    s = env.solver()
    s.set_stream(net.stream.cuda_stream)
    s.store_agents(agents["sec"], agents["sat"], agents["upt"], agents["nex"], np.zeros_like(agents["sec"]), None,
                   agents["vol"], agents["pos"])
    f1 = field[0]
    s.store_densities_device(f1)
    s.run_steps(16, 0)
    s.synchronize()
    e0, e1 = events()
    e0.record(net.stream)
    s.run_steps(160, 16)
    e1.record(net.stream)
    s.synchronize()
    ms_plain16 = e0.elapsed_time(e1) / 10
    s.close()
    with torch.cuda.stream(net.stream):
        out1 = torch.empty_like(f1)
    for _ in range(3):
        run_net.infer(f1, src[0], sink[0], out1)
    run_net.synchronize()
    e0, e1 = events()
    e0.record(net.stream)
    for _ in range(10):
        run_net.infer(f1, src[0], sink[0], out1)
    e1.record(net.stream)
    run_net.synchronize()
    ms_macro = e0.elapsed_time(e1) / 10

    # the trained network rolled out alone for 8 macro-steps from a field and agents of its training
    # distribution (uniform agents), against plain stepping: its relative L2 error after each
    rollout = []
    ua = su.random_agents(env, np.random.default_rng(17), 55_000)
    dev_ua = {k: torch.from_numpy(np.ascontiguousarray(v, np.float32)).cuda() for k, v in ua.items()}
    torch.cuda.synchronize()
    s = env.solver()
    s.set_stream(net.stream.cuda_stream)
    s.store_agents(ua["sec"], ua["sat"], ua["upt"], ua["nex"], np.zeros_like(ua["sec"]), None, ua["vol"], ua["pos"])
    with torch.cuda.stream(net.stream):  # every step below in order on the network's stream
        g_field, g_src, g_sink = [torch.empty((1, VS), device="cuda") for _ in range(3)]
        su.random_field(env.grid, env.S, np.random.default_rng(19), g_field[0], net.stream)
        su.agent_rates((0, 0, 0), (env.dx,) * 3, env.grid, env.time_step, dev_ua, g_src[0], g_sink[0], net.stream)
        s.store_densities_device(g_field[0])
        sur_field = g_field[0].clone()
        plain_now = torch.empty_like(sur_field)
        for m in range(8):
            run_net.infer(sur_field, g_src[0], g_sink[0], out1)
            sur_field.copy_(out1)
            s.run_steps(16, 16 * m)
            s.load_densities_device(plain_now)
            rollout.append(su.rel_l2(sur_field, plain_now))
    s.synchronize()
    s.close()

    # the controller over 1,600 steps, from a field of the training distribution
    run_field = f1.clone()
    report = su.run_with_fallback(run_net, env, run_field, agents, macro_steps=fallback_macro_steps, check_every=8,
                                  tolerance=1e-3)
    s = env.solver()
    s.store_agents(agents["sec"], agents["sat"], agents["upt"], agents["nex"], np.zeros_like(agents["sec"]), None,
                   agents["vol"], agents["pos"])
    s.store_densities_device(f1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.run_steps(16 * fallback_macro_steps, 0)
    s.synchronize()
    plain_s = time.perf_counter() - t0
    plain_field = torch.empty_like(f1)
    s.load_densities_device(plain_field)
    s.synchronize()
    s.close()
    run_net.close()
    net.close()
    gen.close()
    return {
        "VS": VS, "ms_macro": ms_macro, "ms_plain16": ms_plain16, "ms_train": ms_train,
        "train_tflops": train_flop / (ms_train / 1e3) / 1e12, "pairs_per_s": 1.0 / pair_s, "trained": trained,
        "ms_conv": ms_conv, "conv_tflops": achieved, "peak": peak, "peak_kind": peak_kind,
        "fallback_run": {"macro_steps": report.macro_steps, "surrogate_macro_steps": report.surrogate_steps,
                         "checks": [[m, e] for m, e in report.checks], "fell_back_at": report.fell_back_at,
                         "seconds": report.seconds, "plain_seconds": plain_s,
                         "speedup_vs_plain": plain_s / report.seconds,
                         "rel_l2_vs_plain": su.rel_l2(run_field, plain_field)},
        "rollout_rel_l2_uniform_agents": rollout,
    }


def run_surrogate(args):
    """The learned surrogate at 128^3 x 4: training throughput, one convolution against the tensor
    peak, a macro-step against 16 plain steps, and the fallback controller over 1,600 steps."""
    if args.conv_only:
        from parabiofvm_b200 import surrogate as su

        return surrogate_conv_only(args, su.standard_environment())
    r = measure_surrogate(train_steps=max(args.steps, 3), warmup=args.warmup,
                          fresh_train_steps=args.surrogate_train_steps)
    line = {
        "metric": METRIC, "value": r["VS"] * 16 / (r["ms_macro"] / 1e3), "unit": UNIT, "n_gpus": 1, "steps": 10,
        "warmup": 3, "ms_per_step": r["ms_macro"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 weights/activations, f32 accumulate", "data": "synthetic (seeded)",
        "config": {"workload": f"surrogate-128: {SURROGATE_TEXT}", "l2": "activations 4x the L2 at batch 4"},
        "macro_step": {"ms": r["ms_macro"], "plain_16_steps_ms": r["ms_plain16"],
                       "speedup_vs_plain": r["ms_plain16"] / r["ms_macro"]},
        "training": {"ms_per_step_batch4": r["ms_train"], "tflops": r["train_tflops"],
                     "pairs_per_s_generated": r["pairs_per_s"], "network": r["trained"]},
        "roofline": {"bound": "tensor", "kernel": "sur_conv_kernel (forward, batch 4)", "achieved": r["conv_tflops"],
                     "peak": r["peak"], "unit": "TFLOP/s", "frac": r["conv_tflops"] / r["peak"],
                     "peak_kind": r["peak_kind"], "traffic": None, "ms": r["ms_conv"]},
        "fallback_run": r["fallback_run"],
        "rollout_rel_l2_uniform_agents": r["rollout_rel_l2_uniform_agents"],
        "gpu_launches": None,
    }
    print(json.dumps(line), flush=True)
    return 0


def time_sur_conv(grid, B, reps=10, wgrad=False):
    """Device time of one convolution (or weight gradient) launch on [B][grid][32] bf16 tensors."""
    import ctypes

    import torch

    from parabiofvm_b200 import _abi

    lib = _abi.load()
    V = grid[0] * grid[1] * grid[2]
    xin = torch.randn((B, V, 32), device="cuda").to(torch.bfloat16)
    w = (torch.randn((27, 32, 32), device="cuda") * 0.05).to(torch.bfloat16)
    yout = torch.empty_like(xin)
    dW = torch.zeros((27, 32, 32), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    shape = (ctypes.c_int32 * 4)(*grid, B)
    stream = torch.cuda.current_stream()
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

    def once():
        if wgrad:
            _abi.check(lib.bfvm_sur_conv3d_wgrad(shape, p(xin), p(yout), p(dW), p(err),
                                                 ctypes.c_void_p(stream.cuda_stream)))
        else:
            _abi.check(lib.bfvm_sur_conv3d(shape, p(xin), p(w), None, None, 0, None, p(yout), None, None, 0, p(err),
                                           ctypes.c_void_p(stream.cuda_stream)))

    for _ in range(3):
        once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        once()
    e1.record(stream)
    torch.cuda.synchronize()
    if int(err.item()):
        raise RuntimeError("a surrogate kernel timed out")
    return e0.elapsed_time(e1) / reps


def surrogate_conv_only(args, env):
    """The forward convolution and the weight gradient alone (profiling size: --conv-batch)."""
    B = args.conv_batch
    flop = 2.0 * 27 * 32 * 32 * env.voxels * B
    peak, peak_kind = measured_tensor_peak()
    out = {}
    for name, wg in (("conv", False), ("wgrad", True)):
        ms = time_sur_conv(env.grid, B, reps=args.steps, wgrad=wg)
        out[name] = {"ms": ms, "tflops": flop / (ms / 1e3) / 1e12, "frac": flop / (ms / 1e3) / 1e12 / peak}
    print(json.dumps({"workload": f"surrogate-128 convolutions, batch {B}", "peak_tflops": peak,
                      "peak_kind": peak_kind, **out}), flush=True)
    return 0


def run_zslab(args):
    """The plain-320 mesh split along z: one slab per rank (NCCL), or --slabs slabs on one GPU."""
    import torch
    import torch.distributed as dist

    from parabiofvm_b200 import slabs as sl
    from parabiofvm_b200.workloads import make_solver

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local_rank))
    t_setup = time.perf_counter()
    w = make_workload("plain-320")  # one mesh: the same seed on every rank
    count = world if world > 1 else args.slabs
    bounds = sl.plan_slabs(w.grid[2], count)
    mine = [rank] if world > 1 else list(range(count))
    stream = torch.cuda.Stream()
    parts = [sl.make_slab(w, bounds, k, device=local_rank, stream=stream) for k in mine]
    exchange = sl.GroupExchange() if world > 1 else sl.LocalExchange()
    log(f"rank {rank}: slabs {mine} of {bounds} built in {time.perf_counter() - t_setup:.1f}s")

    def barrier():
        if world > 1:
            dist.barrier()

    sl.run_steps(parts, exchange, args.warmup, 0)
    torch.cuda.synchronize()
    sampler = ClockSampler(physical_gpu_index(local_rank))
    sampler.start()
    time.sleep(1.0)
    barrier()
    torch.cuda.synchronize()
    launches0 = sum(p.launch_count for p in parts)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    sl.run_steps(parts, exchange, args.steps, args.warmup)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    launches = sum(p.launch_count for p in parts) - launches0
    ms = reduce_max_over_ranks(ev0.elapsed_time(ev1), world, "cuda")
    VS = w.voxel_count * w.S
    value = VS * args.steps / (ms / 1e3)

    single = None
    if world == 1:
        # the same mesh in one solver on the same GPU, the same steps: the cost of the split, and
        # the agreement of the two (the split z sweep rounds differently)
        s = make_solver(w, device=local_rank)
        s.set_stream(stream.cuda_stream)
        s.run_steps(args.warmup, 0)
        s.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s.run_steps(args.steps, args.warmup)
        b.record(stream)
        torch.cuda.synchronize()
        ms_single = a.elapsed_time(b)
        ref = s.load_densities()
        s.close()
        got = np.concatenate([p.load_densities() for p in parts])
        single = {"ms_per_step": ms_single / args.steps, "value": VS * args.steps / (ms_single / 1e3),
                  "split_overhead": ms / ms_single,
                  "rel_l2_vs_single": _rel_l2(got, ref), "max_rel_vs_single": _max_rel(got, ref)}
    for p in parts:
        p.close()
    if rank == 0:
        peak, peak_kind = measured_peak()
        step_bytes = algorithmic_step_bytes(w)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": f"zslab-320: {WORKLOADS['plain-320']['text']}; split along z into {count} slabs "
                                   f"at planes {bounds}" + (" (one per rank, NCCL exchanges)" if world > 1 else
                                                            " on one GPU (exchanges as copies)"),
                       "slabs": count, "l2": "field 17x the L2, no flush"},
            "step_hbm": {"algorithmic_bytes": step_bytes, "achieved_gbs": step_bytes / (ms / args.steps / 1e3) / 1e9,
                         "frac": step_bytes / (ms / args.steps / 1e3) / 1e9 / peak, "peak_gbs": peak,
                         "peak_kind": peak_kind},
            "single_solver": single,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        log(f"note: WORLD_SIZE={world} differs from --gpus {args.gpus}; using WORLD_SIZE")
    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local_rank))

    from parabiofvm_b200.workloads import make_solver

    t_setup = time.perf_counter()
    w = make_workload(args.workload, seed_offset=rank)
    log(f"rank {rank}: workload built in {time.perf_counter() - t_setup:.1f}s")
    stream = torch.cuda.Stream()
    s = make_solver(w, device=local_rank)
    s.set_stream(stream.cuda_stream)
    for opt in args.option:
        name, val = opt.split("=", 1)
        s.set_option(name, int(val))
    tuned = s.autotune() if args.autotune else None
    VS = w.voxel_count * w.S

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_max_over_ranks(x, world, "cuda")

    def run_steps(n, first):
        if not args.eager:
            s.run_steps(n, first)  # graph replay
            return
        for i in range(n):  # the same kernels, launched one by one
            s.diffusion_gradient()
            s.secretion((first + i) % 10 == 0)

    # ---- device-resident steps
    run_steps(args.warmup, 0)
    s.synchronize()
    sampler = ClockSampler(physical_gpu_index(local_rank))
    sampler.start()
    time.sleep(1.0)  # nvidia-smi needs a moment before its first sample
    barrier()
    torch.cuda.synchronize()
    launches0 = s.launch_count
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    run_steps(args.steps, args.warmup)
    ev1.record(stream)
    s.synchronize()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    launches = s.launch_count - launches0
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = whole_job_rate(world, VS, args.steps, ms)

    # ---- per-kernel timing on the same stream (the roofline numerator); --kernel-reps 0 leaves
    # it out (launch lists of the steps alone)
    kernels, roofline = {}, None
    peak, peak_kind = measured_peak()
    if args.kernel_reps > 0:
        kernels = {}
        reps = args.kernel_reps

        def timed(fn):
            fn()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(reps):
                fn()
            b.record(stream)
            torch.cuda.synchronize()
            return a.elapsed_time(b) / reps

        # the sweeps alone: the Dirichlet conditions are lifted while they are timed, then put back
        # and their overwrite is timed on its own
        for dim in range(w.dims):
            for is_max in (0, 1):
                s.set_boundary_dirichlet(dim, is_max, None, None)
        s.set_interior_dirichlet(np.zeros((0, w.dims), np.int32), np.zeros((0, w.S), np.float32),
                                 np.zeros((0, w.S), bool))
        names = ["sweep_x", "sweep_y", "sweep_z"]
        for axis in range(w.dims):
            kernels[names[axis]] = {"ms": timed(lambda: s.sweep(axis)), "bytes": 8 * VS}
        # the three sweeps with the gradient inside the z sweep (option fused_gradient): the z sweep
        # with its gradient is that time less the x and y sweeps
        if w.dims == 3:
            s.set_option("fused_gradient", 1)
            ms_dg = timed(s.diffusion_gradient)
            s.set_option("fused_gradient", 0)
            kernels["sweep_z_with_gradient_inside"] = {
                "ms": ms_dg - kernels["sweep_x"]["ms"] - kernels["sweep_y"]["ms"], "bytes": (8 + 12) * VS,
                "how": "bfvm_diffusion_gradient_solve with the option fused_gradient, less the x and y sweeps"}
        for (dim, is_max), (vals, conds) in w.boundary.items():
            s.set_boundary_dirichlet(dim, is_max, vals, conds)
        if w.interior_voxels is not None:
            s.set_interior_dirichlet(w.interior_voxels, w.interior_values, w.interior_conditions)
        n_dir = dirichlet_elements(w)
        kernels["dirichlet"] = {"ms": timed(s.dirichlet), "bytes": 16 * n_dir}
        kernels["gradient"] = {"ms": timed(s.gradient), "bytes": (4 + 4 * w.dims) * VS}
        A = w.agents.count
        kernels["secretion"] = {"ms": timed(lambda: s.secretion(False)),
                                "bytes": A * w.S * (12 + 8 + (20 if w.compute_internalized else 0))}
        kernels["secretion_rebin"] = {"ms": timed(lambda: s.secretion(True)), "bytes": None}
        # a whole non-recompute step (graph replay) as configured by default (the Dirichlet scatters and
        # the gradient kernel), then with the Dirichlet overwrites written by the sweeps, then with the
        # gradient inside the z sweep as well
        kernels["step"] = {"ms": timed(lambda: s.run_steps(1, 11)), "bytes": None}
        s.set_option("fused_dirichlet", 1)
        kernels["step_fused_dirichlet"] = {"ms": timed(lambda: s.run_steps(1, 11)), "bytes": None}
        s.set_option("fused_gradient", 1)
        kernels["step_fused_dirichlet_gradient"] = {"ms": timed(lambda: s.run_steps(1, 11)), "bytes": None}
        s.set_option("fused_dirichlet", 0)
        s.set_option("fused_gradient", 0)
        s.synchronize()
        peak, peak_kind = measured_peak()
        for k in kernels.values():
            k["gbs"] = (k["bytes"] / (k["ms"] / 1e3) / 1e9) if k["bytes"] else None
        sweeps = [kernels[n] for n in names[:w.dims]]
        sweep_ms = sum(k["ms"] for k in sweeps) / len(sweeps)
        kernels["sweep_mean"] = {"ms": sweep_ms, "bytes": 8 * VS, "gbs": 8 * VS / (sweep_ms / 1e3) / 1e9}
        traffic_rec = committed_traffic().get(args.workload, {})
        # the dominant kernel: the sweep kernel (three launches per step, the largest share of the
        # step's launch list); its achieved bandwidth is the per-launch algorithmic bytes over the mean
        # launch time
        roofline = {"bound": "hbm", "kernel": "sweep_tma_kernel (mean of the x, y, z launches)",
                    "achieved": 8 * VS / (sweep_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                    "traffic": traffic_rec.get("sweep"), "peak_source": f"{peak_kind} hbm_gbs (copy)",
                    "algorithmic_bytes_per_launch": 8 * VS, "ms_per_launch": sweep_ms}
        roofline["frac"] = roofline["achieved"] / peak
    step_bytes = algorithmic_step_bytes(w)
    step_gbs = step_bytes / (ms / args.steps / 1e3) / 1e9
    step_hbm = {"algorithmic_bytes": step_bytes, "achieved_gbs": step_gbs, "frac_of_measured": step_gbs / peak,
                "frac_of_8000": step_gbs / 8000.0}

    # ---- end to end through the C ABI with pinned host buffers
    e2e = None
    if not args.skip_e2e:
        pinned = lambda n: torch.empty(n, dtype=torch.float32, pin_memory=True).numpy()  # noqa: E731
        field_in = pinned(VS)
        field_in[:] = w.densities
        a = w.agents
        ag = {}
        for key in ("secretion_rates", "saturation_densities", "uptake_rates", "net_export_rates", "internalized",
                    "fraction_released", "volumes", "positions"):
            arr = np.asarray(getattr(a, key), np.float32).reshape(-1)
            ag[key] = pinned(arr.size)
            ag[key][:] = arr
        field_out = pinned(VS)
        grad_out = pinned(VS * w.dims)
        intern_out = pinned(A * w.S)
        pos_step = pinned(A * w.dims)
        pos_step[:] = np.asarray(a.positions, np.float32).reshape(-1)
        # once: the state in and out, as the reference's device solver stores it before its loop and
        # loads it after (densities and internalized substrates: src/solver/device/CUDA/
        # device_context.cpp:99-116); every step: the agents' positions in and their internalized
        # substrates out.  The gradients stay on the device; loading them too is timed after.
        h2d = field_in.nbytes + sum(v.nbytes for v in ag.values()) + args.steps * pos_step.nbytes
        d2h = field_out.nbytes + args.steps * intern_out.nbytes
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.store_densities(field_in)
        s.store_agents(ag["secretion_rates"], ag["saturation_densities"], ag["uptake_rates"], ag["net_export_rates"],
                       ag["internalized"], ag["fraction_released"], ag["volumes"], ag["positions"])
        for k in range(args.steps):
            # the agents' copies run on the solver's copy stream and overlap the step's diffusion;
            # the step (one graph launch) waits for them right before its secretion
            s.store_agent_positions_async(pos_step)
            s.run_steps(1, k)
            s.load_internalized_async(intern_out)
        s.load_densities(field_out)
        s.synchronize()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1))
        # the gradients loaded as well (6.3 GB at plain-320), for comparison
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        s.load_gradients(grad_out)
        g1.record(stream)
        torch.cuda.synchronize()
        grad_ms = max_over_ranks(g0.elapsed_time(g1))
        e2e = {"value": whole_job_rate(world, VS, args.steps, e2e_ms), "unit": UNIT,
               "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps,
               "ms_total": e2e_ms,
               "with_gradients_loaded": {"value": whole_job_rate(world, VS, args.steps, e2e_ms + grad_ms),
                                         "gradient_load_ms": grad_ms,
                                         "d2h_bytes_per_step": (d2h + grad_out.nbytes) // args.steps},
               "what": "through the C ABI from pinned host memory: field and agents stored before the steps, "
                       "every step the agents' positions stored, the step run (bfvm_run_steps: diffusion, gradient, "
                       "secretion) and the internalized substrates loaded (the per-step copies asynchronous, "
                       "overlapping the step's diffusion), the field loaded after the steps (the reference device "
                       "solver's store/load set); with_gradients_loaded adds loading the gradients"}
        del field_in, field_out, grad_out, intern_out, ag

    s.close()
    del s
    torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        rate, threads, times = cpu_oracle_rate(w, budget_s=args.cpu_budget_s)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "cpu_model": host_cpu_model(), "kind": "port",
               "sample": f"{len(times)} full step(s) of the same workload on {threads} host threads "
                         f"({', '.join(f'{t:.2f}s' for t in times)})"}

    parity = None
    if rank == 0 and world == 1 and not args.skip_parity:
        t_par = time.perf_counter()
        parity = [parity_report(args.workload, 1, with_fp64=False), parity_report("plain-50", 100, with_fp64=True)]
        log(f"parity checks took {time.perf_counter() - t_par:.1f}s")

    extras = {}
    if rank == 0 and world == 1 and not args.skip_extras:
        t_ex = time.perf_counter()
        extras = side_forms()
        log(f"batch and surrogate measurements took {time.perf_counter() - t_ex:.1f}s")

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    w_text = WORKLOADS[args.workload]["text"]
    line = {
        "options": args.option + ([f"autotuned sweep shapes (groups, stages) per axis: {tuned}"] if tuned else []),
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"{args.workload}: {w_text}", "grid": list(w.grid), "substrates": w.S,
                   "agents": w.agents.count,
                   "interior_dirichlet_voxels": 0 if w.interior_voxels is None else len(w.interior_voxels),
                   "l2": "inputs larger than L2 (2.1 GB field per sweep), no flush" if VS * 4 > 126e6 else
                         "L2-resident parity workload",
                   "parallelism": f"{world} independent replica(s), one per GPU"},
        "roofline": roofline,
        "step_hbm": step_hbm,
        "kernels": kernels,
        "cpu_baseline": cpu,
        "parity": parity,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clocks,
        **extras,
    }
    print(json.dumps(line), flush=True)
    return 0


def side_forms():
    """The two forms that stand beside the plain step, measured briefly on the same GPU after it:
    ``batch_256`` (10 batched steps against the same instances stepped alone) and ``surrogate_128``
    (a macro-step of the trained network against 16 plain steps, the convolution against the tensor
    peak, and the fallback controller over 1,600 steps)."""
    out = {}
    b = measure_batch(10, 3, clocks=False)
    units = b["voxel_substrates"]
    out["batch_256"] = {
        "workload": f"batch-256: {BATCH_TEXT}", "steps": 10, "warmup": 3,
        "ms_per_step": b["ms_batch"] / 10, "value": units * 10 / (b["ms_batch"] / 1e3), "unit": UNIT,
        "sequential_ms_per_step": b["ms_sequential"] / 10,
        "speedup_vs_sequential": b["ms_sequential"] / b["ms_batch"],
        "max_rel_l2_vs_alone": b["max_rel_l2_vs_alone"], "autotuned": b["autotuned"], "gpu_launches": b["launches"]}
    r = measure_surrogate(train_steps=5, warmup=3)
    fb = r["fallback_run"]
    out["surrogate_128"] = {
        "workload": f"surrogate-128: {SURROGATE_TEXT}",
        "macro_step_ms": r["ms_macro"], "plain_16_steps_ms": r["ms_plain16"],
        "macro_step_speedup_vs_plain": r["ms_plain16"] / r["ms_macro"],
        "conv_tflops": r["conv_tflops"], "conv_frac_of_peak": r["conv_tflops"] / r["peak"], "peak_kind": r["peak_kind"],
        "train_step_ms_batch4": r["ms_train"], "network": r["trained"],
        "controller": {"macro_steps": fb["macro_steps"], "surrogate_macro_steps": fb["surrogate_macro_steps"],
                       "checked_rel_l2": fb["checks"], "fell_back_at": fb["fell_back_at"],
                       "speedup_vs_plain": fb["speedup_vs_plain"], "rel_l2_vs_plain": fb["rel_l2_vs_plain"]},
        "rollout_rel_l2_uniform_agents": r["rollout_rel_l2_uniform_agents"]}
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["batch-256", "zslab-320", "surrogate-128"],
                    default="plain-320")
    ap.add_argument("--parity-steps", type=int, default=0,
                    help="only compare the GPU with the FP32 and FP64 oracles over this many steps")
    ap.add_argument("--conv-only", action="store_true",
                    help="surrogate-128: time the convolution kernels alone (profiling)")
    ap.add_argument("--conv-batch", type=int, default=4)
    ap.add_argument("--surrogate-train-steps", type=int, default=100,
                    help="surrogate-128: Adam steps on fresh pairs before the controller runs")
    ap.add_argument("--slabs", type=int, default=2,
                    help="zslab-320 in one process: slabs emulated on the one GPU")
    ap.add_argument("--kernel-reps", type=int, default=5)
    ap.add_argument("--option", action="append", default=[],
                    help="solver tuning option name=value (bfvm_set_option), e.g. tma_sweeps=0")
    ap.add_argument("--eager", action="store_true",
                    help="launch each step's kernels one by one instead of replaying the step's CUDA graph")
    ap.add_argument("--autotune", action="store_true",
                    help="measure the sweeps' launch shapes before timing (bfvm_autotune)")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-parity", action="store_true",
                    help="leave out the oracle comparisons (one full-size step, 100 steps of plain-50)")
    ap.add_argument("--skip-extras", action="store_true",
                    help="leave out the brief batch-256 and surrogate-128 measurements of the default line")
    ap.add_argument("--cpu-budget-s", type=float, default=20.0)
    ap.add_argument("--reference-budget-s", type=float, default=150.0)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        log("warm-up raised to 3 steps")
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.parity_steps:
        print(json.dumps(step_parity(args.workload, args.parity_steps)), flush=True)
        return 0
    if args.workload == "batch-256":
        return run_batch(args)
    if args.workload == "zslab-320":
        return run_zslab(args)
    if args.workload == "surrogate-128":
        return run_surrogate(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
