#!/usr/bin/env python
"""Throughput of the explicit central-difference stepper in element-cycles/s.

Workload (headline): the large elastic-plastic block -- 256x128x64 8-node
hexahedra (2,097,152 elements, 2,154,945 nodes), J2 plasticity, seeded
smoothed-Gaussian initial velocities, bottom face fixed, 5000 cycles.  One
bench step is ``--cycles-per-step`` cycles (default 500) of the stepper on
the resident model.  The per-cycle working set (1.2-2.4 GB) is far larger
than the 126 MB L2, so no flush is needed between timed steps.  ``value`` is
the headline precision (default mixed); the other precision is timed the
same way beside it.

Accuracy (``fp64_vs_mixed``): fresh FP64 and mixed steppers run exactly the
workload's 5000 cycles (``--accuracy-cycles``) from the same initial state,
whatever --steps and --warmup are; the mixed result's maximum relative
displacement error and energy-balance drift against FP64 at that point are
the headline accuracy figures.  The same two figures after all the cycles
the timed runs made are reported beside them (``after_timed_cycles``).

End to end (``e2e``, and ``e2e_fp64`` beside the mixed headline): through
the C ABI with host buffers; every step uploads the state from pinned host
memory, runs the step's cycles and reads u, v and sigma back, over --steps
steps.

Further legs of the same run (one GPU):
  batched_block  the block workload as a one-instance batch, mixed and FP64
                 (the batched engine's own rate on the headline mesh);
  batched_sweep  256 uneven cantilever/plate instances (2k-60k elements, own
                 material, dt and clock), 3000 cycles each, in one mixed
                 batch and in one FP64 batch (every instance's mixed error
                 and energy drift against its FP64 run; the maximum is
                 reported), with both batches' cycle bytes against the
                 copy peak (``cycle_roofline``); the plain FP64 stepper
                 solves a sample of them one after another; the reference
                 CPU stepper solves a sample as one process per instance on
                 all host cores (``cpu_reference``);
  serving        a seeded Poisson stream (50/s, 500 requests) of
                 1k-500k-element solves served with continuous batching
                 under a 150 GB budget: solves/s and p50/p99 latency; the
                 first 100 requests also through the plain FP64 stepper one
                 at a time (latency, and each result's mixed error and
                 energy drift against FP64), and alone through the same
                 server; attached to it, the deck-reading time of the
                 reference reader and DataInFast on a 500,000-element deck
                 (``deck_read``) and output written while the device steps
                 against output written synchronously (``output_overlap``).

Arms:
  --impl ours (default)  the sm_100a stepper through the C ABI
                         (enscdynamics_b200/_lib/libensc_b200.so)
  --impl reference       the reference CPU stepper (compiled from its sources
                         into oracle/_ref) on a bounded slab of the same
                         workload, at the fastest of 1, 2, 4, 8 and all host
                         threads

One JSON line is printed by rank 0.  Multi-GPU (torchrun): every rank runs
an independent replica of the block workload (the stepper has no
cross-instance exchange), so scaling is weak and ``value`` sums all ranks'
element-cycles over the slowest rank's device time.  The sweep's instances
are sharded across the ranks (every world-th instance per rank, no
collective on the data path); the serving stream is sharded the same way
by request (every rank serves every world-th request on its own GPU; the
outcomes are gathered for the stream's percentiles), and its comparisons
with the sequential FP64 stepper run at one GPU only.
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
    ap.add_argument("--accuracy-cycles", type=int, default=5000,
                    help="cycles of the fresh FP64-vs-mixed comparison (the block workload's 5000; 0: skip)")
    ap.add_argument("--e2e-steps", type=int, default=0, help="steps of the end-to-end legs (0: --steps)")
    ap.add_argument("--cpu-cycles", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweep-instances", type=int, default=256, help="batched sweep leg (0: skip)")
    ap.add_argument("--sweep-cycles", type=int, default=3000)
    ap.add_argument("--sweep-fp64-sample", type=int, default=32)
    ap.add_argument("--serve-requests", type=int, default=500, help="serving leg (0: skip)")
    ap.add_argument("--batched-block-cycles", type=int, default=1024,
                    help="timed cycles of the block as a one-instance batch, each precision (0: skip)")
    ap.add_argument("--serve-seq-sample", type=int, default=100,
                    help="requests of the serving stream also served by the plain FP64 stepper one at a time")
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


def element_pass_bytes(ne: int, nn: int, plastic: bool, mixed: bool = False, patches: int = 0,
                       partials: int = 0) -> int:
    """Algorithmic bytes of one element-pass launch.
    FP64: connectivity 32, sigma r/w 96, QIA r/w 192, B0^T 192, V0 8,
    element-force write 192 per element (+16 eps_p r/w with J2); x, u, v
    gathered once per node (72 B).
    Mixed: connectivity 32, sigma r/w 48, QIA r/w 96, the B0 matrix A as a
    float pair 72, V0 8, cbrt(V0) 4 (+8 eps_p) per element; x FP64 and v
    FP32 per node (36 B: the mixed pass forms F from current coordinates and
    does not read u).  Slot assembly: force write 96 per element.  Patch
    assembly (partials > 0): the incidence list 16 per element, per
    (patch, node) partial its incidence offset 4 and its three FP32 sums 12,
    and 4 per patch for the partial range -- instead of the force write."""
    if mixed:
        base = ne * (32 + 48 + 96 + 72 + 8 + 4 + (8 if plastic else 0)) + nn * 36
        if partials:
            return base + ne * 16 + partials * (4 + 12) + (patches + 1) * 4
        return base + ne * 96
    return ne * (32 + 96 + 192 + 192 + 8 + 192 + (16 if plastic else 0)) + nn * 72


def node_pass_bytes(ne: int, nn: int, mixed: bool = False, partials: int = 0) -> int:
    """Algorithmic bytes of one node-pass launch: the element forces, and
    per node the inverse mass 8, BC code 1, x and u read and write 96 (mixed:
    x only, 48 -- the mixed stepper keeps x - u in the u rows and forms u
    when the state is read), v read and write (48 FP64; mixed: 24 for the
    float rows and 12 for their 16-bit residual rows).  Slot assembly: the 24 force components of every element,
    each read once (192 B FP64, 96 B mixed).  Patch assembly (partials > 0):
    per node its partial range 4, per partial its index 4 and its three sums
    12.  Reactions and prescribed velocities are touched only at constrained
    nodes and not counted; slot-major force slots that no element fills
    (boundary nodes) are read as zeros but not counted."""
    if mixed:
        per_node = nn * (8 + 1 + 48 + 24 + 12)
        if partials:
            return per_node + nn * 4 + partials * (4 + 12)
        return ne * 96 + per_node
    return ne * 192 + nn * (8 + 1 + 96 + 48)


def cycle_bytes(ne: int, nn: int, plastic: bool, mixed: bool = False, patches: int = 0, partials: int = 0) -> int:
    """Canonical algorithmic bytes of one cycle (element pass + node pass):
    FP64 904 B per element (+16 with J2) and 225 B per node; mixed with the
    slot assembly 452 B per element (+8) and 129 B per node; mixed with the
    patch assembly 276 B per element (+8), 133 B per node and 32 B per
    partial (about 1.5-1.8 partials per node)."""
    return (element_pass_bytes(ne, nn, plastic, mixed, patches, partials)
            + node_pass_bytes(ne, nn, mixed, partials))


def build_problem(name: str, dims: str = "256,128,64"):
    from enscdynamics_b200 import workloads
    if name == "block":
        nx, ny, nz = (int(v) for v in dims.split(","))
        return workloads.block(nx, ny, nz, 1.0 * nx / 256, 0.5 * ny / 128, 0.25 * nz / 64)
    return workloads.cantilever()


# --------------------------------------------------------------------------
# CPU legs (reference stepper compiled from its sources; checker territory)

def thread_counts() -> list:
    """Thread counts the CPU legs try: 1, 2, 4, 8 and all host threads."""
    n = os.cpu_count() or 1
    return sorted({t for t in (1, 2, 4, 8, n) if t <= n})


class CpuReference:
    """The reference CPU stepper (compiled from its own sources into
    oracle/_ref) on a slab of the block workload: the deck is written once,
    each run parses it, sets up and times its cycle loop.  More OpenMP
    threads are not always faster for the reference (its parallel regions
    and per-cycle zeroing cost more than they save at this size), so the
    legs time every count of ``thread_counts`` briefly and use the fastest."""

    def __init__(self):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle
        from enscdynamics_b200 import workloads
        self.pyoracle = pyoracle
        self.ok = pyoracle.harness_available()
        self.dir = tempfile.mkdtemp(prefix="ensc_ref_")
        self.deck = None
        if self.ok:
            nx, ny, nz = CPU_SAMPLE_DIMS
            self.p = workloads.block(nx, ny, nz, 1.0, 0.5, 0.25 * nz / 64, plastic=False)
            self.deck = self.p.write_deck(self.dir)
            self.elements = self.p.mesh.n_elements

    def run(self, cycles: int, threads: int) -> dict:
        r = self.pyoracle.run_reference(self.dir, self.deck, "time", cycles, threads=threads)
        r["value"] = self.elements * cycles / r["loop_s"]
        return r

    def choose_threads(self, cycles: int = 3):
        """(fastest thread count, {threads: element-cycles/s}) over a short run each."""
        rates = {t: self.run(cycles, t)["value"] for t in thread_counts()}
        return max(rates, key=rates.get), rates

    def sample_text(self, cycles: int, threads: int) -> str:
        nx, ny, nz = CPU_SAMPLE_DIMS
        return (f"{nx}x{ny}x{nz} slab ({self.elements} elements) of the block workload, elastic (the reference "
                f"has no J2), {cycles} cycles per run, cycle loop timed by the harness, OMP_NUM_THREADS={threads} "
                f"(fastest of {thread_counts()})")

    def close(self):
        import shutil
        shutil.rmtree(self.dir, ignore_errors=True)


def cpu_sweep_leg(sweep_cycles: int, sample: int = 16, cycles: int = 40) -> dict:
    """The reference CPU stepper on the batched sweep, solved the way the
    reference can solve many instances at once: one process per instance
    (its solver state is process-wide), one OpenMP thread each, as many
    concurrent processes as host cores.  A bounded sample: the first `sample`
    instances of the sweep (elastic: the reference has no J2), `cycles`
    cycles each, all started together; solves/s extrapolates each instance's
    cycle loop to the sweep's cycle count and adds its parse and setup."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from concurrent.futures import ThreadPoolExecutor
    from enscdynamics_b200 import workloads as W
    if not pyoracle.harness_available():
        return {"unavailable": "reference harness not built (oracle/_ref)"}
    cores = os.cpu_count() or 1
    n = max(1, min(sample, cores))
    probs = [W.sweep_instance(i, cycles=sweep_cycles) for i in range(n)]
    dirs = [tempfile.mkdtemp(prefix="ensc_sweep_ref_") for _ in probs]
    try:
        decks = [q.write_deck(d) for q, d in zip(probs, dirs)]
        t0 = time.perf_counter()
        with ThreadPoolExecutor(n) as pool:
            runs = list(pool.map(lambda a: pyoracle.run_reference(a[0], a[1], "time", cycles, threads=1),
                                 zip(dirs, decks)))
        wall = time.perf_counter() - t0
    finally:
        import shutil
        for d in dirs:
            shutil.rmtree(d, ignore_errors=True)
    solve_s = [r["parse_s"] + r["loop_s"] * sweep_cycles / cycles for r in runs]
    work = sum(q.mesh.n_elements for q in probs) * cycles
    return {"processes": n, "cores": cores, "sample": f"first {n} sweep instances, elastic, {cycles} cycles each",
            "solves_per_s": n / statistics.mean(solve_s) if n else 0.0,
            "element_cycles_per_s": work / max(r["loop_s"] for r in runs), "wall_s": wall}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    ref = CpuReference()
    if not ref.ok:
        print(json.dumps({"impl": "reference", "unavailable": "reference harness not built (oracle/_ref)"}))
        return 0
    t0 = time.time()
    try:
        # warm-up: every thread count once, keep the fastest
        threads, rates = ref.choose_threads(max(2, args.cpu_cycles // 8))
        for _ in range(max(0, args.warmup - 1)):
            ref.run(max(2, args.cpu_cycles // 4), threads)
        runs = [ref.run(args.cpu_cycles, threads) for _ in range(args.steps)]
    finally:
        ref.close()
    wall = time.time() - t0
    loop = [r["loop_s"] for r in runs]
    value = ref.elements * args.cpu_cycles * len(runs) / sum(loop)
    sample = ref.sample_text(args.cpu_cycles, threads)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sum(loop) / len(loop),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "block 256x128x64 hex8 J2 (reference sample: elastic slab)",
                       "elements": ref.elements, "cycles_per_step": args.cpu_cycles, "threads": threads},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "reference",
                             "sample": sample, "by_threads": rates},
            "parse_s": statistics.median(r["parse_s"] for r in runs),
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
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
    asm = s.assembly
    pt, pq = asm["patches"], asm["partials"]
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
    el_bytes = element_pass_bytes(ne, nn, plastic, mixed, pt, pq)
    nd_bytes = node_pass_bytes(ne, nn, mixed, pq)
    achieved = el_bytes / (el_ms / 1000.0) / 1e9
    total_ms = sum(v["ms"] for v in prof.values())
    traffic = None
    tp = os.path.join(ROOT, "profiles", f"element_{precision}_block_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get("bytes_per_launch")
    cb = cycle_bytes(ne, nn, plastic, mixed, pt, pq)
    kernel = ("k_element_mixed_patch" if pq else "k_element_mixed_staged") if mixed else "k_element_fp64_warp"
    return s, {
        "assembly": {"kind": "patch" if pq else "slot", "patches": pt, "partials": pq},
        "value": value, "ms_max": ms_max, "launches": args.steps * (C * kpc + 1),
        "clocks": clocks, "cycles_run": (args.warmup + args.steps) * C + args.profile_cycles,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "kernel": "element pass (%s)" % kernel,
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
    step's input state (x, u, v, sigma, QIA, eps_p and the clock) from pinned
    host memory, runs C cycles, and reads back u, v and sigma into pinned
    host memory; timed with CUDA events around all steps."""
    import ctypes as C_
    import numpy as np
    import torch
    C = args.cycles_per_step
    steps = args.e2e_steps or args.steps
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
    for _ in range(steps):
        s._check(lib.ensc_upload_state(s.h, ptr(pin["x"]), ptr(pin["u"]), ptr(pin["v"]), ptr(pin["sigma"]),
                                       ptr(pin["qia"]), ptr(pin["eps_p"]), clk["time"], clk["dt_i"], clk["dt_i_1"],
                                       clk["dt_stable_min"]))
        s.step_async(C)
        s._check(lib.ensc_download(s.h, None, ptr(outp["u"]), ptr(outp["v"]), ptr(outp["sigma"]), None, None))
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    value = replica_value(float(s.n_elements) * C * steps, ms, max_over_ranks, sum_over_ranks)
    return {"value": value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": steps,
            "ms_per_step": max_over_ranks(ms) / steps}


def energy_balance(e: dict) -> float:
    """kinetic + internal + hourglass + viscous - external work."""
    return e["kinetic"] + e["internal"] + e["hourglass"] + e["viscous"] - e["external"]


def compare_to_fp64(u_mixed, u_fp64, e_mixed: dict, e_fp64: dict) -> dict:
    """The accuracy bars of the mixed stepper against FP64 on the same solve:
    max |u_mixed - u_fp64| / max |u_fp64|, and the energy-balance drift
    |E_bal(mixed) - E_bal(FP64)| / KE0."""
    import numpy as np
    umax = float(np.abs(u_fp64).max())
    err = float(np.abs(u_mixed - u_fp64).max() / umax) if umax > 0 else float(np.abs(u_mixed).max())
    ke0 = e_fp64["kinetic0"]
    drift = abs(energy_balance(e_mixed) - energy_balance(e_fp64)) / ke0 if ke0 > 0 else 0.0
    return {"max_rel_disp_err": err, "energy_drift": drift}


def accuracy_leg(args, p, local, stream) -> dict:
    """Fresh FP64 and mixed steppers on the block workload, each run exactly
    ``--accuracy-cycles`` cycles (the workload's 5000) from the same initial
    state, independent of --steps / --warmup; the mixed result's
    displacement error and energy drift against FP64 (compare_to_fp64), and
    how far each run's energy balance moved from its initial kinetic energy
    (|E_bal - KE0| / KE0)."""
    import numpy as np
    from enscdynamics_b200 import capi
    cyc = args.accuracy_cycles
    nn = p.mesh.n_nodes
    out = {}
    for prec in (capi.FP64, capi.MIXED):
        with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls, device=local,
                          stream=stream.cuda_stream, precision=prec) as s:
            s.set_bcs(p.bc_code, p.bc_value)
            rep = s.step(cyc)
            assert rep["status"] == 0 and rep["cycles"] == cyc, rep
            out[prec] = (s.download({"u": np.empty((nn, 3))})["u"], s.energy(), rep["time"])
    (u64, e64, t64), (umx, emx, tmx) = out[capi.FP64], out[capi.MIXED]
    r = compare_to_fp64(umx, u64, emx, e64)
    r.update({"cycles": cyc, "time_fp64": t64, "time_mixed": tmx,
              "energy_balance_fp64": abs(energy_balance(e64) - e64["kinetic0"]) / e64["kinetic0"],
              "energy_balance_mixed": abs(energy_balance(emx) - emx["kinetic0"]) / emx["kinetic0"],
              "bars": {"max_rel_disp_err": 1e-5, "energy_drift": 5e-3}})
    r["pass"] = r["max_rel_disp_err"] <= 1e-5 and r["energy_drift"] <= 5e-3
    return r


def shard(n: int, world: int, rank: int) -> list:
    """The instances of an n-instance workload that rank `rank` of `world`
    runs: every world-th one, so that ranks get similar mixes of sizes."""
    return list(range(rank, n, world))


def batched_block_leg(args, local, p) -> dict:
    """The block workload through the batched engine, one instance per
    batch, mixed and FP64: after the autotuner's runs (700 cycles),
    args.batched_block_cycles cycles timed with CUDA events; then 64 more
    cycles inside an NVTX range named batched_block_<precision>, for a
    kernel launch list of the batched passes."""
    import torch
    from enscdynamics_b200 import capi
    stream = torch.cuda.Stream()
    out = {}
    for prec, name in ((capi.MIXED, "mixed"), (capi.FP64, "fp64")):
        with capi.Batch(max_instances=1, max_elements=p.mesh.n_elements, max_nodes=p.mesh.n_nodes,
                        budget_bytes=100 * 10 ** 9, precision=prec, device=local, stream=stream.cuda_stream) as b:
            sl = b.add(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls)
            b.set_bcs(sl, p.bc_code, p.bc_value)
            b.arm(sl, 10 ** 9)
            b.run(700)
            b.sync()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.run(args.batched_block_cycles)
            e1.record(stream)
            b.sync()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / args.batched_block_cycles
            torch.cuda.nvtx.range_push(f"batched_block_{name}")
            b.run(64)
            b.sync()
            torch.cuda.nvtx.range_pop()
            cb = cycle_bytes(p.mesh.n_elements, p.mesh.n_nodes, True, prec == capi.MIXED)
            out[name] = {"element_cycles_per_s": p.mesh.n_elements / (ms / 1000.0), "ms_per_cycle": ms,
                         "cycle_frac": cb / (ms / 1000.0) / 1e9 / measured_peaks()[0], "tuning": b.tuning}
    out["mixed_over_batched_fp64"] = out["mixed"]["element_cycles_per_s"] / out["fp64"]["element_cycles_per_s"]
    return out


def sweep_leg(args, local, world=1, rank=0, barrier=lambda: None, max_over_ranks=lambda x: x,
              sum_over_ranks=lambda x: x):
    """Batched parameter sweep: args.sweep_instances uneven instances, each
    its own material, dt and clock, args.sweep_cycles cycles each, in one
    batch in mixed precision, timed with CUDA events from the first run to
    the last instance's completion.  The same instances then run as one
    FP64 batch (timed the same way), which gives every instance's mixed
    displacement error and energy drift against FP64 (the maximum over
    instances is reported); and the plain FP64 stepper solves a bounded
    sample of them one after another.  With several ranks the instances are
    sharded across them (shard), each rank runs its share in its own
    batches, and the rates are totals over the slowest rank's time."""
    import torch
    from enscdynamics_b200 import capi
    from enscdynamics_b200 import workloads as W
    n, cyc = args.sweep_instances, args.sweep_cycles
    mine = shard(n, world, rank)
    probs = [W.sweep_instance(i, cycles=cyc) for i in mine]
    ne_tot = sum(p.mesh.n_elements for p in probs)
    nn_tot = sum(p.mesh.n_nodes for p in probs)
    stream = torch.cuda.Stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def run_batch(precision):
        t0 = time.perf_counter()
        b = capi.Batch(max_instances=len(probs), max_elements=ne_tot, max_nodes=nn_tot, budget_bytes=150 * 10 ** 9,
                       precision=precision, device=local, stream=stream.cuda_stream)
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
        e0.record(stream)
        b.run(cyc)
        e1.record(stream)
        running = b.sync()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        assert running == 0
        reps = [b.report(sl) for sl in slots]
        bad = [i for i, r in enumerate(reps) if r["status"] != 0 or r["cycles"] != cyc]
        res = [(b.download(sl, ("u",))["u"], b.energy(sl)) for sl in slots]
        tuning = b.tuning
        b.close()
        return {"ms": max_over_ranks(ms), "admit_s": admit_s, "device_bytes": dev_bytes, "bad": len(bad),
                "tuning": tuning, "res": res}

    mx = run_batch(capi.MIXED)
    f64 = run_batch(capi.FP64)
    acc = [compare_to_fp64(um, u64, em, e64) for (um, em), (u64, e64) in zip(mx["res"], f64["res"])]
    worst_err = max_over_ranks(max(a["max_rel_disp_err"] for a in acc))
    worst_drift = max_over_ranks(max(a["energy_drift"] for a in acc))
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
    ms = mx["ms"]
    batched = n / (ms / 1000.0)
    seq = sum_over_ranks(k / (seq_ms / 1000.0))
    rate_mx = ne_all * cyc / (ms / 1000.0)
    rate_64 = ne_all * cyc / (f64["ms"] / 1000.0)
    # the cycle bytes of all instances (the batched passes run the J2 update
    # for every instance), over the batch's time, against the copy peak
    peak, peak_kind = measured_peaks()
    bytes_mx = sum_over_ranks(float(sum(cycle_bytes(p.mesh.n_elements, p.mesh.n_nodes, True, True) for p in probs)))
    bytes_64 = sum_over_ranks(float(sum(cycle_bytes(p.mesh.n_elements, p.mesh.n_nodes, True) for p in probs)))
    gbs_mx = bytes_mx * cyc / (ms / 1000.0) / 1e9
    gbs_64 = bytes_64 * cyc / (f64["ms"] / 1000.0) / 1e9
    return {"instances": n, "cycles": cyc, "elements": int(ne_all), "ranks": world,
            "elements_range": [min(p.mesh.n_elements for p in probs), max(p.mesh.n_elements for p in probs)],
            "precision": "mixed", "solves_per_s": batched, "element_cycles_per_s": rate_mx,
            "ms": ms, "admit_s": mx["admit_s"], "device_bytes": mx["device_bytes"],
            "failed": int(sum_over_ranks(float(mx["bad"] + f64["bad"]))),
            "tuning": mx["tuning"],
            "accuracy_vs_fp64": {"max_rel_disp_err": worst_err, "energy_drift": worst_drift,
                                 "instances": n, "of": "maximum over instances"},
            "batched_fp64": {"element_cycles_per_s": rate_64, "solves_per_s": n / (f64["ms"] / 1000.0),
                             "ms": f64["ms"], "tuning": f64["tuning"]},
            "mixed_over_batched_fp64": rate_mx / rate_64,
            "cycle_roofline": {"mixed_gbs": gbs_mx, "mixed_frac": gbs_mx / peak, "fp64_gbs": gbs_64,
                               "fp64_frac": gbs_64 / peak, "peak": peak, "peak_source": peak_kind,
                               "nodes_per_element": float(sum_over_ranks(float(nn_tot))) / ne_all},
            "sequential_fp64": {"sample": int(sum_over_ranks(float(k))), "solves_per_s": seq,
                                "element_cycles_per_s": sum_over_ranks(seq_work / (seq_ms / 1000.0))},
            "speedup_vs_sequential_fp64": batched / seq}


def deck_read_leg(elements_per_side=(100, 100, 50)) -> dict:
    """Deck reading time at the serving stream's largest request size: a
    500,000-element block deck with per-node initial velocities, read by the
    reference's DataIn and by DataInFast (ensc_reader_bench, built with the
    drop-in), which must fill the solver identically."""
    exe = os.path.join(ROOT, "enscdynamics_b200", "_lib", "ensc_reader_bench")
    if not os.path.exists(exe):
        return {"unavailable": "ensc_reader_bench not built (needs the reference sources)"}
    from enscdynamics_b200 import workloads as W
    nx, ny, nz = elements_per_side
    p = W.block(nx, ny, nz, 0.004 * nx, 0.004 * ny, 0.004 * nz, plastic=False)
    with tempfile.TemporaryDirectory() as d:
        deck = p.write_deck(d)
        r = subprocess.run([exe, os.path.join(d, deck), "2"], cwd=d, capture_output=True, text=True, timeout=600)
    if r.returncode not in (0, 3):
        return {"unavailable": "ensc_reader_bench failed: " + r.stderr[-300:]}
    out = json.loads(r.stdout.strip().splitlines()[-1])
    out.pop("deck", None)
    out["deck"] = f"block {nx}x{ny}x{nz} with per-node initial velocities (best of 2 reads each)"
    return out


def output_leg(local, frames: int = 6, interval: int = 1000, dims=(128, 64, 32)) -> dict:
    """Output written while the device steps (ensc_snapshot_begin /
    ensc_step_until_async / ensc_snapshot_wait, the drop-in's output
    pattern), mixed precision on a 128x64x32 block (262,144 elements):
    `frames` output intervals of `interval` cycles, at each output time the
    fields x, u, v, a, reactions and sigma are encoded as base64, as the .vtu
    writer does.  (a) no output; (b) output overlapped: begin the snapshot,
    enqueue the next interval, then take and encode the snapshot while it
    runs; (c) output written synchronously: run the interval, download,
    encode.  Both write the same snapshot fields; the snapshot buffers are
    allocated before timing.  Wall times; hidden = (c - b) / (c - a), the
    share of the output cost that overlapping takes off the critical path."""
    import base64
    import numpy as np
    import torch
    from enscdynamics_b200 import capi
    from enscdynamics_b200 import workloads as W
    nx, ny, nz = dims
    p = W.block(nx, ny, nz, 1.0 * nx / 256, 0.5 * ny / 128, 0.25 * nz / 64)
    stream = torch.cuda.Stream()

    def encode(fields):
        return sum(len(base64.b64encode(np.ascontiguousarray(v).tobytes())) for v in fields.values()
                   if isinstance(v, np.ndarray))

    times = {}
    with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls, device=local,
                      stream=stream.cuda_stream, precision=capi.MIXED) as s:
        s.set_bcs(p.bc_code, p.bc_value)
        s.step(interval)
        s.snapshot_begin()  # allocates the device and pinned snapshot buffers
        s.snapshot_wait()
        enc = 0
        for mode in ("none", "overlapped", "synchronous", "none_again"):
            s.step(1)  # a force pass since the last download
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(frames):
                if mode.startswith("none"):
                    s.step_async(interval)
                    s.sync()
                elif mode == "overlapped":
                    s.snapshot_begin()
                    s.step_until_async(interval, math.inf, math.inf)
                    enc += encode(s.snapshot_wait())
                    s.sync()
                else:
                    s.step_async(interval)
                    s.sync()
                    s.snapshot_begin()
                    enc += encode(s.snapshot_wait())
            torch.cuda.synchronize()
            times[mode] = time.perf_counter() - t0
    a = min(times["none"], times["none_again"])
    b, c = times["overlapped"], times["synchronous"]
    return {"elements": p.mesh.n_elements, "frames": frames, "cycles_per_frame": interval,
            "no_output_s": a, "overlapped_s": b, "synchronous_s": c,
            "hidden": (c - b) / (c - a) if c > a else None, "encoded_bytes": enc,
            "fields": "x, u, v, a, reactions, sigma"}


def gather_outcomes(outcomes, world: int) -> list:
    """Every rank's serving outcomes on every rank (all_gather of plain
    tuples; identity at one rank), rebuilt as Outcome objects."""
    from enscdynamics_b200 import serving as S
    rows = [(o.index, o.arrival, o.admitted, o.finished, o.cycles, o.status, o.elements) for o in outcomes]
    if world > 1:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, rows)
        rows = [r for part in parts for r in part]
    out = [S.Outcome(i, a, admitted=ad, finished=f, cycles=c, status=st, elements=e) for i, a, ad, f, c, st, e in rows]
    return sorted(out, key=lambda o: o.index)


def serve_leg_ranks(args, local, world: int, rank: int, barrier) -> dict:
    """The serving stream over several GPUs: the same seeded stream, every
    world-th request served by this rank's own loop and batch on its own GPU
    (instances are independent, so no collective on the data path); the
    outcomes are gathered for the whole stream's solves/s and latency
    percentiles."""
    from enscdynamics_b200 import serving as S
    from enscdynamics_b200 import workloads as W
    reqs = W.serving_requests(args.serve_requests, rate=50.0, seed=11)
    mine = [r for r in reqs if r.index % world == rank]
    workers = max(1, min(4, (os.cpu_count() or 2) // max(1, world) - 1))
    be = S.BatchBackend(budget_bytes=150 * 10 ** 9, max_instances=1024, device=local, fields=())
    srv = S.Server(be, prepare_workers=workers)
    barrier()  # the ranks start the stream together
    try:
        out = srv.serve(mine)
    finally:
        be.close()
    summ = S.summarize(gather_outcomes(out, world))
    summ.update({"rate_per_s": 50.0, "budget_bytes_per_gpu": 150 * 10 ** 9, "precision": "mixed", "ranks": world,
                 "sharding": "request i on rank i mod world"})
    return summ


def serve_leg(args, local):
    """Serving stream: args.serve_requests Poisson arrivals at 50/s, element
    counts log-uniform in 1k-500k, 1000-10000 cycles, elastic or J2, mixed
    precision, admitted against a 150 GB device budget, with the host part of
    each admission prepared on worker threads while the GPU steps.  Beside
    it, the first args.serve_seq_sample requests of the same stream (a) served
    alone by the same loop and (b) through the plain FP64 stepper one request
    at a time (each request's solve time measured; its queueing follows from
    the arrivals, and the first k requests' latencies in a one-at-a-time
    server depend only on those k), so that (a) and (b) face the same k
    requests.  The FP64 results of that sample give each sampled request's
    mixed displacement error and energy drift (maximum over the sample
    reported)."""
    import numpy as np
    import torch
    from enscdynamics_b200 import capi
    from enscdynamics_b200 import serving as S
    from enscdynamics_b200 import workloads as W
    reqs = W.serving_requests(args.serve_requests, rate=50.0, seed=11)
    workers = max(1, min(4, (os.cpu_count() or 2) - 1))

    def serve(rs):
        be = S.BatchBackend(budget_bytes=150 * 10 ** 9, max_instances=1024, device=local, fields=("u",))
        srv = S.Server(be, prepare_workers=workers)
        try:
            res = srv.serve(rs)
        finally:
            be.close()
        return res, {k: (round(v, 3) if isinstance(v, float) else v) for k, v in srv.stats.items()}

    out, host = serve(reqs)
    summ = S.summarize(out)
    k = min(len(reqs), args.serve_seq_sample)
    alone, _ = serve(reqs[:k])
    first_alone = S.summarize(alone)
    # sequential FP64: solve times per request, queue by arrival
    stream = torch.cuda.Stream()
    fin = 0.0
    lat = []
    work = 0
    acc = []
    t_first = reqs[0].arrival
    for r, o in zip(reqs[:k], out[:k]):
        p = r.problem
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls, device=local,
                          stream=stream.cuda_stream, precision=capi.FP64) as s:
            s.set_bcs(p.bc_code, p.bc_value)
            s.step(p.cycles)
            u64 = s.download({"u": np.empty((p.mesh.n_nodes, 3))})["u"]
            e64 = s.energy()
        dt = time.perf_counter() - t0
        start = max(r.arrival, fin)
        fin = start + dt
        lat.append(fin - r.arrival)
        work += p.mesh.n_elements * p.cycles
        if o.status == 0:
            acc.append(compare_to_fp64(o.result["u"], u64, o.energy, e64))
    span = fin - t_first
    seq = {"requests": k, "solves_per_s": k / span, "p50_latency_s": float(np.percentile(lat, 50)),
           "p99_latency_s": float(np.percentile(lat, 99)), "element_cycles_per_s": work / span}
    summ.update({"rate_per_s": 50.0, "budget_bytes": 150 * 10 ** 9, "precision": "mixed",
                 "prepare_workers": workers, "host_time_s": host,
                 "first_k_alone": {kk: first_alone[kk] for kk in ("requests", "makespan_s", "solves_per_s",
                                                                  "p50_latency_s", "p99_latency_s",
                                                                  "element_cycles_per_s", "failed")},
                 "accuracy_vs_fp64": {"max_rel_disp_err": max(a["max_rel_disp_err"] for a in acc),
                                      "energy_drift": max(a["energy_drift"] for a in acc),
                                      "requests": len(acc), "of": f"maximum over the first {k} requests"},
                 "sequential_fp64": seq,
                 "vs_sequential_fp64": {
                     "first_k_solves_per_s": first_alone["solves_per_s"] / seq["solves_per_s"],
                     "first_k_p99_latency": seq["p99_latency_s"] / first_alone["p99_latency_s"],
                     "stream_solves_per_s": summ["solves_per_s"] / seq["solves_per_s"],
                     "of": "ratios > 1 favour the batched mixed server; stream_solves_per_s sets the whole "
                           "stream's rate against the sequential rate on its first k requests"}})
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
    e2e_other = None
    if not args.single_precision:
        s_other, m_other = time_block(args, p, other, stream, local, barrier, max_over_ranks, sum_over_ranks)
        # the two timed steppers ran the same cycles from the same state: the
        # mixed result's accuracy after all the cycles the timing ran
        st = {}
        for name, s in ((head, s_head), (other, s_other)):
            st[name] = (s.download({"u": np.empty((nn, 3))})["u"], s.energy())
        after = compare_to_fp64(st["mixed"][0], st["fp64"][0], st["mixed"][1], st["fp64"][1])
        after["cycles"] = m_head["cycles_run"]
        e2e_other = e2e_block(args, s_other, stream, max_over_ranks, sum_over_ranks, barrier)
        s_other.close()
        m64, mmx = (m_other, m_head) if head == "mixed" else (m_head, m_other)
        cmp = {"fp64_value": m64["value"], "mixed_value": mmx["value"],
               "mixed_over_fp64": mmx["value"] / m64["value"],
               "fp64_roofline_frac": m64["roofline"]["frac"], "mixed_roofline_frac": mmx["roofline"]["frac"],
               "fp64_node_roofline_frac": m64["node_roofline"]["frac"],
               "after_timed_cycles": after}
        if args.workload == "block" and args.accuracy_cycles > 0:
            acc = accuracy_leg(args, p, local, stream)
            cmp["at_workload_cycles"] = acc
            # the headline accuracy figures: the workload's own cycle count
            cmp["mixed_max_rel_disp_err"] = acc["max_rel_disp_err"]
            cmp["mixed_energy_drift"] = acc["energy_drift"]
            cmp["cycles_compared"] = acc["cycles"]
    e2e = e2e_block(args, s_head, stream, max_over_ranks, sum_over_ranks, barrier)
    s_head.close()

    sweep = serve = bblock = None
    if rank == 0 and world == 1 and args.batched_block_cycles > 0 and args.workload == "block":
        bblock = batched_block_leg(args, local, p)
        if cmp is not None:
            bblock["mixed_over_plain_fp64"] = bblock["mixed"]["element_cycles_per_s"] / cmp["fp64_value"]
    if args.sweep_instances > 0:
        sweep = sweep_leg(args, local, world, rank, barrier, max_over_ranks, sum_over_ranks)
    if args.serve_requests > 0:
        serve = serve_leg(args, local) if world == 1 else serve_leg_ranks(args, local, world, rank, barrier)
        if rank == 0:
            serve["deck_read"] = deck_read_leg()
            serve["output_overlap"] = output_leg(local)

    if sweep is not None and rank == 0 and world == 1 and not args.no_cpu_baseline:
        sweep["cpu_reference"] = cpu_sweep_leg(args.sweep_cycles)
        if sweep["cpu_reference"].get("solves_per_s"):
            sweep["speedup_vs_cpu_reference"] = sweep["solves_per_s"] / sweep["cpu_reference"]["solves_per_s"]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref = CpuReference()
        if ref.ok:
            try:
                threads, rates = ref.choose_threads()
                r = ref.run(args.cpu_cycles, threads)
            finally:
                ref.close()
            cpu = {"value": r["value"], "unit": METRIC, "cores": threads, "kind": "reference",
                   "sample": ref.sample_text(args.cpu_cycles, threads), "by_threads": rates,
                   "parse_s": r["parse_s"]}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    mixed = head == "mixed"
    steps_text = (f"{C} cycles per step, {args.steps} timed steps after {args.warmup} warm-up steps "
                  f"({(args.warmup + args.steps) * C} cycles per stepper); accuracy of mixed against FP64 at the "
                  f"workload's {args.accuracy_cycles} cycles from a fresh start")
    if args.workload == "block":
        dims = "x".join(args.block_dims.split(","))
        workload = f"block {dims} hex8 ({ne:,} el, {nn:,} nodes), J2; {steps_text}"
    else:
        workload = p.name
    line = {
        "metric": METRIC, "value": m_head["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": m_head["ms_max"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if mixed else "f64", "data": "synthetic",
        "config": {"workload": workload, "elements": ne, "nodes": nn, "cycles_per_step": C, "precision": head,
                   "l2": f"inputs larger than L2 ({m_head['cycle_roofline']['bytes_per_cycle'] / 1e9:.2f} GB "
                         "per cycle)",
                   "parallelism": f"replicas x{world}"},
        "assembly": m_head["assembly"],
        "roofline": m_head["roofline"],
        "node_roofline": m_head["node_roofline"],
        "cycle_roofline": m_head["cycle_roofline"],
        "kernel_share": m_head["kernel_share"],
        "fp64_vs_mixed": cmp,
        "batched_block": bblock,
        "batched_sweep": sweep,
        "serving": serve,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "e2e_" + other: e2e_other,
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
