#!/usr/bin/env python
"""Throughput of the explicit central-difference stepper in element-cycles/s.

Workload (headline): the large elastic-plastic block -- 256x128x64 8-node
hexahedra (2,097,152 elements, 2,154,945 nodes), J2 plasticity, seeded
smoothed-Gaussian initial velocities, bottom face fixed.  One bench step is
``--cycles-per-step`` cycles (default 500) of the stepper on the resident
model; ten steps make the workload's 5000 cycles.  The per-cycle working set
(1.3-2.3 GB) is far larger than the 126 MB L2, so no flush is needed between
timed steps.  ``value`` is the headline precision (default mixed); the other
precision is timed the same way beside it, and the mixed result's maximum
displacement error against FP64 after the same cycles is reported.

Further legs of the same run (one GPU):
  batched_sweep  256 uneven cantilever/plate instances (2k-60k elements, own
                 material, dt and clock), 3000 cycles each, in one batch;
                 solves/s beside the plain FP64 stepper solving a sample of
                 them one after another;
  serving        a seeded Poisson stream (50/s) of 1k-500k-element solves
                 served with continuous batching under a 150 GB budget;
                 solves/s and p50/p99 latency beside the plain FP64 stepper
                 serving the same stream one request at a time.

Arms:
  --impl ours (default)  the sm_100a stepper through the C ABI
                         (enscdynamics_b200/_lib/libensc_b200.so)
  --impl reference       the reference CPU stepper (compiled from its sources
                         into oracle/_ref) on a bounded slab of the same
                         workload, with all host threads

One JSON line is printed by rank 0.  Multi-GPU (torchrun): every rank runs
an independent replica of the block workload (the stepper has no
cross-instance exchange), so scaling is weak and ``value`` sums all ranks'
element-cycles over the slowest rank's device time.  The sweep's instances
are sharded across the ranks (every world-th instance per rank, no
collective on the data path); the serving leg runs at one GPU only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "element-cycles/s"
CPU_SAMPLE_DIMS = (256, 128, 8)      # slab of the block workload for the CPU legs


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["block", "cantilever"], default="block")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed",
                    help="precision of the headline number; the other one is measured beside it")
    ap.add_argument("--single-precision", action="store_true", help="measure the headline precision only")
    ap.add_argument("--cycles-per-step", type=int, default=500)
    ap.add_argument("--block-dims", default="256,128,64", help="block workload cells nx,ny,nz")
    ap.add_argument("--profile-cycles", type=int, default=40)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-cycles", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweep-instances", type=int, default=256, help="batched sweep leg (0: skip)")
    ap.add_argument("--sweep-cycles", type=int, default=3000)
    ap.add_argument("--sweep-fp64-sample", type=int, default=32)
    ap.add_argument("--serve-requests", type=int, default=48, help="serving leg (0: skip)")
    return ap.parse_args()


# --------------------------------------------------------------------------
# helpers

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.uuid}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def element_pass_bytes(ne: int, nn: int, plastic: bool, mixed: bool = False) -> int:
    """Algorithmic bytes of one element-pass launch.
    FP64: connectivity 32, sigma r/w 96, QIA r/w 192, B0^T 192, V0 8,
    element-force write 192 per element (+16 eps_p r/w with J2); x, u, v
    gathered once per node (72 B).
    Mixed: connectivity 32, sigma r/w 48, QIA r/w 96, the B0 matrix A as a
    float pair 72, V0 8, cbrt(V0) 4, force write 96 (+8 eps_p); x FP64 and
    v FP32 per node (36 B: the mixed pass forms F from current coordinates
    and does not read u)."""
    if mixed:
        return ne * (32 + 48 + 96 + 72 + 8 + 4 + 96 + (8 if plastic else 0)) + nn * 36
    return ne * (32 + 96 + 192 + 192 + 8 + 192 + (16 if plastic else 0)) + nn * 72


def node_pass_bytes(ne: int, nn: int, mixed: bool = False) -> int:
    """Algorithmic bytes of one node-pass launch: the element forces (24
    components per element, each read once: 192 B FP64, 96 B mixed), and per
    node the inverse mass 8, BC code 1, x and u read and write 96, v read and
    write (48 FP64, 24 mixed).  Reactions and prescribed velocities are
    touched only at constrained nodes and not counted; force slots that no
    element fills (boundary nodes) are read as zeros but not counted."""
    if mixed:
        return ne * 96 + nn * (8 + 1 + 96 + 24)
    return ne * 192 + nn * (8 + 1 + 96 + 48)


def cycle_bytes(ne: int, nn: int, plastic: bool, mixed: bool = False) -> int:
    """Canonical algorithmic bytes of one cycle (element pass + node pass):
    FP64 904 B per element (+16 with J2) and 225 B per node; mixed 452 B per
    element (+8) and 165 B per node."""
    return element_pass_bytes(ne, nn, plastic, mixed) + node_pass_bytes(ne, nn, mixed)


def build_problem(name: str, dims: str = "256,128,64"):
    from enscdynamics_b200 import workloads
    if name == "block":
        nx, ny, nz = (int(v) for v in dims.split(","))
        return workloads.block(nx, ny, nz, 1.0 * nx / 256, 0.5 * ny / 128, 0.25 * nz / 64)
    return workloads.cantilever()


# --------------------------------------------------------------------------
# CPU legs (reference stepper compiled from its sources; checker territory)

def cpu_reference_sample(cycles: int, threads: int, repeats: int = 1):
    """Times the reference CPU stepper on a slab of the block workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from enscdynamics_b200 import workloads
    if not pyoracle.harness_available():
        return None
    nx, ny, nz = CPU_SAMPLE_DIMS
    p = workloads.block(nx, ny, nz, 1.0, 0.5, 0.25 * nz / 64, plastic=False)
    out = []
    with tempfile.TemporaryDirectory() as d:
        deck = p.write_deck(d)
        for _ in range(repeats):
            r = pyoracle.run_reference(d, deck, "time", cycles, threads=threads)
            out.append(r)
    ne = p.mesh.n_elements
    return {"elements": ne, "cycles": cycles, "runs": out,
            "loop_s": [r["loop_s"] for r in out],
            "value": ne * cycles * len(out) / sum(r["loop_s"] for r in out)}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_reference_sample(max(2, args.cpu_cycles // 4), threads)
    t0 = time.time()
    res = cpu_reference_sample(args.cpu_cycles, threads, repeats=args.steps)
    wall = time.time() - t0
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference harness not built (oracle/_ref)"}))
        return 0
    nx, ny, nz = CPU_SAMPLE_DIMS
    sample = (f"{nx}x{ny}x{nz} slab ({res['elements']} elements) of the block workload, elastic (the reference "
              f"has no J2), {args.cpu_cycles} cycles per step, cycle loop timed by the harness")
    line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * sum(res["loop_s"]) / len(res["loop_s"]),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "block 256x128x64 hex8 J2 (reference sample: slab)", "elements": res["elements"],
                       "cycles_per_step": args.cpu_cycles, "threads": threads},
            "cpu_baseline": {"value": res["value"], "unit": METRIC, "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": res["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------------
# GPU arm

def time_block(args, p, precision, stream, local, barrier, max_over_ranks, sum_over_ranks):
    """Times K steps of C cycles of the block workload on one resident
    stepper; returns the stepper (still open) and the measurements."""
    import torch
    from enscdynamics_b200 import capi
    mixed = precision == "mixed"
    ne, nn = p.mesh.n_elements, p.mesh.n_nodes
    plastic = p.material.yield_stress > 0.0
    C = args.cycles_per_step
    s = capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls, device=local,
                     stream=stream.cuda_stream, precision=capi.MIXED if mixed else capi.FP64)
    s.set_bcs(p.bc_code, p.bc_value)
    kpc = s.kernels_per_cycle
    for _ in range(args.warmup):
        s.step_async(C)
    s.sync()
    uuid = str(torch.cuda.get_device_properties(local).uuid)
    if not uuid.startswith("GPU-"):
        uuid = "GPU-" + uuid
    sampler = ClockSampler(uuid)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        s.step_async(C)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    ms = ev0.elapsed_time(ev1)
    rep = s.sync()
    assert rep["status"] == 0, rep
    ms_max = max_over_ranks(ms)
    value = replica_value(float(ne) * C * args.steps, ms, max_over_ranks, sum_over_ranks)
    # per-kernel CUDA-event durations on the launching stream (roofline)
    prof = s.profile(args.profile_cycles)
    el = prof["element"]
    el_ms = el["ms"] / max(el["launches"], 1)
    nd = prof["node"]
    nd_ms = nd["ms"] / max(nd["launches"], 1)
    peak, peak_kind = measured_peaks()
    el_bytes = element_pass_bytes(ne, nn, plastic, mixed)
    nd_bytes = node_pass_bytes(ne, nn, mixed)
    achieved = el_bytes / (el_ms / 1000.0) / 1e9
    total_ms = sum(v["ms"] for v in prof.values())
    traffic = None
    tp = os.path.join(ROOT, "profiles", f"element_{precision}_block_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get("bytes_per_launch")
    cb = cycle_bytes(ne, nn, plastic, mixed)
    return s, {
        "value": value, "ms_max": ms_max, "launches": args.steps * (C * kpc + 1),
        "clocks": clocks, "cycles_run": (args.warmup + args.steps) * C + args.profile_cycles,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "kernel": "element pass (%s)" % ("k_element_mixed_staged" if mixed else "k_element_staged, FP64"),
                     "peak_source": peak_kind, "kernel_ms": el_ms, "bytes_per_launch": el_bytes},
        "node_roofline": {"achieved": nd_bytes / (nd_ms / 1000.0) / 1e9, "frac": nd_bytes / (nd_ms / 1000.0) / 1e9 / peak,
                          "kernel_ms": nd_ms, "bytes_per_launch": nd_bytes},
        "cycle_roofline": {"bytes_per_cycle": cb,
                           "achieved_gbs": cb * C * args.steps / (ms_max / 1000.0) / 1e9,
                           "frac": cb * C * args.steps / (ms_max / 1000.0) / 1e9 / peak},
        "kernel_share": {k: v["ms"] / total_ms for k, v in prof.items()},
    }


def e2e_block(args, s, stream, max_over_ranks, sum_over_ranks, barrier):
    """End to end through the C ABI with host buffers: each step uploads the
    step's input state from pinned host memory, runs C cycles, and reads back
    u, v and sigma into pinned host memory."""
    import ctypes as C_
    import numpy as np
    import torch
    C = args.cycles_per_step
    ck = s.download()
    clk = s.step(0)
    pin = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in ck.items()}
    outp = {k: torch.empty(pin[k].shape, dtype=torch.float64).pin_memory() for k in ("u", "v", "sigma")}
    h2d = sum(int(t.numel() * 8) for t in pin.values())
    d2h = sum(int(t.numel() * 8) for t in outp.values())
    P = C_.POINTER(C_.c_double)
    ptr = lambda t: C_.cast(t.data_ptr(), P)  # noqa: E731
    lib = s._lib
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        s._check(lib.ensc_upload_state(s.h, ptr(pin["x"]), ptr(pin["u"]), ptr(pin["v"]), ptr(pin["sigma"]),
                                       ptr(pin["qia"]), ptr(pin["eps_p"]), clk["time"], clk["dt_i"], clk["dt_i_1"],
                                       clk["dt_stable_min"]))
        s.step_async(C)
        s._check(lib.ensc_download(s.h, None, ptr(outp["u"]), ptr(outp["v"]), ptr(outp["sigma"]), None, None))
    e1.record(stream)
    torch.cuda.synchronize()
    value = replica_value(float(s.n_elements) * C * args.e2e_steps, e0.elapsed_time(e1), max_over_ranks,
                          sum_over_ranks)
    return {"value": value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}


def shard(n: int, world: int, rank: int) -> list:
    """The instances of an n-instance workload that rank `rank` of `world`
    runs: every world-th one, so that ranks get similar mixes of sizes."""
    return list(range(rank, n, world))


def sweep_leg(args, local, world=1, rank=0, barrier=lambda: None, max_over_ranks=lambda x: x,
              sum_over_ranks=lambda x: x):
    """Batched parameter sweep: args.sweep_instances uneven instances, each
    its own material, dt and clock, args.sweep_cycles cycles each, in one
    batch (mixed precision).  Timed with CUDA events from the first run to
    the last instance's completion; the plain FP64 stepper solves a bounded
    sample of the same instances one after another for comparison.  With
    several ranks the instances are sharded across them (shard), each rank
    runs its share in its own batch, and the rates are the totals over the
    slowest rank's time."""
    import torch
    from enscdynamics_b200 import capi
    from enscdynamics_b200 import workloads as W
    n, cyc = args.sweep_instances, args.sweep_cycles
    mine = shard(n, world, rank)
    probs = [W.sweep_instance(i, cycles=cyc) for i in mine]
    ne_tot = sum(p.mesh.n_elements for p in probs)
    nn_tot = sum(p.mesh.n_nodes for p in probs)
    stream = torch.cuda.Stream()
    t0 = time.perf_counter()
    b = capi.Batch(max_instances=n, max_elements=ne_tot, max_nodes=nn_tot, budget_bytes=150 * 10 ** 9,
                   precision=capi.MIXED, device=local, stream=stream.cuda_stream)
    slots = []
    for p in probs:
        sl = b.add(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls)
        b.set_bcs(sl, p.bc_code, p.bc_value)
        b.arm(sl, cyc)
        slots.append(sl)
    admit_s = time.perf_counter() - t0
    dev_bytes = b.device_bytes
    torch.cuda.synchronize()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.run(cyc)
    e1.record(stream)
    running = b.sync()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    tuning = b.tuning
    assert running == 0
    bad = [i for i, sl in enumerate(slots) if b.report(sl)["status"] != 0 or b.report(sl)["cycles"] != cyc]
    b.close()
    ms = max_over_ranks(ms)
    # plain FP64 stepper, one solve after another, on a bounded sample
    k = min(len(probs), -(-args.sweep_fp64_sample // world))
    seq_ms = 0.0
    seq_work = 0
    for p in probs[:k]:
        with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls, device=local,
                          stream=stream.cuda_stream, precision=capi.FP64) as s:
            s.set_bcs(p.bc_code, p.bc_value)
            torch.cuda.synchronize()
            e0.record(stream)
            s.step_async(cyc)
            e1.record(stream)
            s.sync()
            torch.cuda.synchronize()
            seq_ms += e0.elapsed_time(e1)
            seq_work += p.mesh.n_elements * cyc
    ne_all = sum_over_ranks(float(ne_tot))
    batched = n / (ms / 1000.0)
    seq = sum_over_ranks(k / (seq_ms / 1000.0))
    return {"instances": n, "cycles": cyc, "elements": int(ne_all), "ranks": world,
            "elements_range": [min(p.mesh.n_elements for p in probs), max(p.mesh.n_elements for p in probs)],
            "precision": "mixed", "solves_per_s": batched, "element_cycles_per_s": ne_all * cyc / (ms / 1000.0),
            "ms": ms, "admit_s": admit_s, "device_bytes": dev_bytes, "failed": int(sum_over_ranks(float(len(bad)))),
            "tuning": tuning,
            "sequential_fp64": {"sample": int(sum_over_ranks(float(k))), "solves_per_s": seq,
                                "element_cycles_per_s": sum_over_ranks(seq_work / (seq_ms / 1000.0))},
            "speedup_vs_sequential_fp64": batched / seq}


def serve_leg(args, local):
    """Serving stream: args.serve_requests Poisson arrivals at 50/s, element
    counts log-uniform in 1k-500k, 1000-10000 cycles, elastic or J2, mixed
    precision, admitted against a 150 GB device budget.  Beside it, the same
    stream through the plain FP64 stepper one request at a time (each
    request's solve time measured; its queueing follows from the arrivals)."""
    import numpy as np
    import torch
    from enscdynamics_b200 import capi
    from enscdynamics_b200 import serving as S
    from enscdynamics_b200 import workloads as W
    reqs = W.serving_requests(args.serve_requests, rate=50.0, seed=11)
    be = S.BatchBackend(budget_bytes=150 * 10 ** 9, max_instances=1024, device=local, fields=("u",))
    try:
        out = S.Server(be).serve(reqs)
    finally:
        be.close()
    summ = S.summarize(out)
    # sequential FP64: solve times per request, queue by arrival
    stream = torch.cuda.Stream()
    fin = 0.0
    lat = []
    work = 0
    t_first = reqs[0].arrival
    for r in reqs:
        p = r.problem
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls, device=local,
                          stream=stream.cuda_stream, precision=capi.FP64) as s:
            s.set_bcs(p.bc_code, p.bc_value)
            s.step(p.cycles)
            s.download({"u": np.empty((p.mesh.n_nodes, 3))})
        dt = time.perf_counter() - t0
        start = max(r.arrival, fin)
        fin = start + dt
        lat.append(fin - r.arrival)
        work += p.mesh.n_elements * p.cycles
    span = fin - t_first
    seq = {"solves_per_s": len(reqs) / span, "p50_latency_s": float(np.percentile(lat, 50)),
           "p99_latency_s": float(np.percentile(lat, 99)), "element_cycles_per_s": work / span}
    summ.update({"rate_per_s": 50.0, "budget_bytes": 150 * 10 ** 9, "precision": "mixed",
                 "sequential_fp64": seq,
                 "speedup_vs_sequential_fp64": summ["solves_per_s"] / seq["solves_per_s"]})
    return summ


def rank_ops(world: int, device):
    """The collective steps of a replica run: a barrier, and the max and the
    sum of one float over all ranks (identity at one rank).  Every rank calls
    them in the same order."""
    import torch
    import torch.distributed as dist

    def barrier():
        if world > 1:
            dist.barrier()

    def reduce(x: float, op) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max_over_ranks(x: float) -> float:
        return reduce(x, dist.ReduceOp.MAX)

    def sum_over_ranks(x: float) -> float:
        return reduce(x, dist.ReduceOp.SUM)

    return barrier, max_over_ranks, sum_over_ranks


def replica_value(work: float, ms: float, max_over_ranks, sum_over_ranks) -> float:
    """Whole-job throughput of a replica run: all ranks' units over the
    slowest rank's device time."""
    return sum_over_ranks(work) / (max_over_ranks(ms) / 1000.0)


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    barrier, max_over_ranks, sum_over_ranks = rank_ops(world, torch.device("cuda", local))

    p = build_problem(args.workload, args.block_dims)
    ne, nn = p.mesh.n_elements, p.mesh.n_nodes
    plastic = p.material.yield_stress > 0.0
    C = args.cycles_per_step
    stream = torch.cuda.Stream()
    head = args.precision
    other = "fp64" if head == "mixed" else "mixed"
    s_head, m_head = time_block(args, p, head, stream, local, barrier, max_over_ranks, sum_over_ranks)
    cmp = None
    if not args.single_precision:
        s_other, m_other = time_block(args, p, other, stream, local, barrier, max_over_ranks, sum_over_ranks)
        # the two steppers ran the same cycles from the same state: the
        # mixed result's displacement error against FP64
        u_h = s_head.download({"u": np.empty((nn, 3))})["u"]
        u_o = s_other.download({"u": np.empty((nn, 3))})["u"]
        s_other.close()
        u64, umx = (u_o, u_h) if head == "mixed" else (u_h, u_o)
        err = float(np.abs(umx - u64).max() / np.abs(u64).max())
        m64, mmx = (m_other, m_head) if head == "mixed" else (m_head, m_other)
        cmp = {"fp64_value": m64["value"], "mixed_value": mmx["value"],
               "mixed_over_fp64": mmx["value"] / m64["value"],
               "mixed_max_rel_disp_err": err, "cycles_compared": m_head["cycles_run"],
               "fp64_roofline_frac": m64["roofline"]["frac"], "mixed_roofline_frac": mmx["roofline"]["frac"]}
    e2e = e2e_block(args, s_head, stream, max_over_ranks, sum_over_ranks, barrier)
    s_head.close()

    sweep = serve = None
    if args.sweep_instances > 0:
        sweep = sweep_leg(args, local, world, rank, barrier, max_over_ranks, sum_over_ranks)
    if world == 1 and args.serve_requests > 0:
        serve = serve_leg(args, local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        res = cpu_reference_sample(args.cpu_cycles, threads)
        one = cpu_reference_sample(max(3, args.cpu_cycles // 4), 1) if res is not None else None
        if res is not None:
            nx, ny, nz = CPU_SAMPLE_DIMS
            cpu = {"value": res["value"], "unit": METRIC, "cores": threads, "kind": "reference",
                   "sample": f"{nx}x{ny}x{nz} slab ({res['elements']} elements) of the block workload, elastic "
                             f"(the reference has no J2), {args.cpu_cycles} cycles, cycle loop timed by the harness",
                   "value_1_thread": one["value"], "sample_1_thread": f"the same slab, {one['cycles']} cycles, "
                                                                      f"OMP_NUM_THREADS=1"}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    mixed = head == "mixed"
    line = {
        "metric": METRIC, "value": m_head["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": m_head["ms_max"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if mixed else "f64", "data": "synthetic",
        "config": {"workload": ("block 256x128x64 hex8 (2,097,152 el, 2,154,945 nodes), J2, 5000 cycles = 10 steps"
                                if args.block_dims == "256,128,64" else p.name) if args.workload == "block" else p.name,
                   "elements": ne, "nodes": nn, "cycles_per_step": C, "precision": head,
                   "l2": f"inputs larger than L2 ({cycle_bytes(ne, nn, plastic, mixed) / 1e9:.2f} GB per cycle)",
                   "parallelism": f"replicas x{world}"},
        "roofline": m_head["roofline"],
        "node_roofline": m_head["node_roofline"],
        "cycle_roofline": m_head["cycle_roofline"],
        "kernel_share": m_head["kernel_share"],
        "fp64_vs_mixed": cmp,
        "batched_sweep": sweep,
        "serving": serve,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": m_head["launches"],
        "clocks": m_head["clocks"],
    }
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
