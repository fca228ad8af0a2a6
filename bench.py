#!/usr/bin/env python
"""Served shower stream on the B200 (one JSON line on rank 0).

Workload (the metric's own configuration): Gaussian synthetic showers of the
seed-21 stream (element count log-uniform in 500-50000, 0.15 m of charged track
per element, vertices uniform in a cylinder of radius 200 m and height 600 m
around the centroid of the 384-OM array, isotropic directions) in the
synthetic Baikal-like water, tables 2-450 m (60 radial nodes), 65 RTE and 321
readout frequencies, 160 bins of 5 ns, threshold 0.01 pe. A step is
``SHOWERS_PER_STEP`` showers; step k takes the next ones from a pool of
``POOL`` distinct showers of the stream.

* ``value``: showers/s of the served mixed-precision path (``ShowerServer``:
  continuous batching over worker streams, split-BF16 readout), every step's
  showers queued at once, element arrays already resident in HBM. Timed with
  CUDA events on the main stream around the whole served region (the workers'
  streams are synchronised inside it).
* ``plain_fp32``: the plain FP32 GPU path, one shower per call
  (``ShowerTransport.__call__``, fp32 readout), on the same showers.
* ``e2e``: the served path through the public API from host element arrays:
  the upload of every step's elements and the read-back of every response
  field inside the timed region.
* ``latency``: p50/p99 from arrival to response under Poisson arrivals at half
  the served rate.
* ``roofline``: the group stage of the fine order 1 (``o1_group_kernel``),
  measured live with the library's kernel timing; ``kernel_times`` lists the
  other timed kernels.
* ``cpu_baseline``: the CPU oracle of the route (float64, one thread per core
  over the OMs) on a bounded sample of the same stream.

``--impl reference`` times that CPU restatement of the reference route on the
host cores, one shower of the stream per step, and prints the same line.
``--gpus N`` under torchrun runs N independent replicas (weak scaling).
The calibration-flash stream (config 1) is measured as an extra key.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "showers/s + p99 latency, served mixed-precision vs plain GPU at <=1e-3 rel pe error"
TABLES = ROOT / "lighthit_b200" / "tables"
FLASH_TABLE = TABLES / "flash_450nm_2-250m.npz"
POOL = 96
SHOWERS_PER_STEP = 16
WORKERS = 3
MAX_BATCH = 8
N_FLASH = 4096
# DRAM bytes (read + write) of one 4096-flash flash_tc_kernel launch, measured with
# ncu on a B200 (profiles/flash_tc_kernel_4096flashes.txt).
FLASH_TC_TRAFFIC = 636_147_456
# DRAM bytes of one o1_group_kernel launch per (OM, pencil) evaluation, from the
# ncu capture of profiles/order1_kernels_16showers_c2.txt (296 MB for 9472 x 256
# threads over (OM, pencil) items), or None when not captured.
O1_GROUP_TRAFFIC_PER_ITEM = None
PENCIL_BYTES = 20 * 8  # one float64 pencil record read per (OM, pencil) evaluation


def max_over_ranks(ms, device):
    """The slowest rank's time (ms): every rank takes the same collective step;
    one rank alone returns its own time."""
    import torch
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return float(ms)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, ms):
    """Whole-job throughput of ``world`` replicas (weak scaling): the units all
    ranks processed over the slowest rank's time."""
    return world * units_per_rank / (ms / 1e3)


def shower_pool(centroid, count=POOL):
    """The first ``count`` showers of the seeded config-2 stream (host dicts)."""
    from lighthit_b200.workloads import gaussian_shower, shower_stream
    draws = shower_stream(count, centroid)
    return [gaussian_shower(d["position_m"], d["direction"],
                            charged_track_length_m=d["charged_track_length_m"],
                            elements=d["elements"], seed=d["seed"]) for d in draws]


def step_showers(pool, k, per_step=SHOWERS_PER_STEP):
    return [pool[(k * per_step + i) % len(pool)] for i in range(per_step)]


def config_json(pool, steps):
    sizes = [len(s["length_m"]) for s in pool]
    return {"workload": "config 2: served stream of Gaussian synthetic showers (seed 21, "
                        "500-50000 elements log-uniform, 0.15 m per element, vertices in a "
                        "200 m x 600 m cylinder, isotropic) on the 384-OM array, tables 2-450 m",
            "showers_per_step": SHOWERS_PER_STEP, "distinct_showers": len(pool),
            "elements_per_shower": {"min": int(min(sizes)), "median": int(np.median(sizes)),
                                    "max": int(max(sizes))},
            "n_om": 384, "omega_nodes": 65, "readout_nodes": 321, "bins": 160,
            "served": {"workers": WORKERS, "max_batch": MAX_BATCH,
                       "readout": "split-bf16 tcgen05 (fp32 accumulate)",
                       ">=2 contraction": "split-bf16 tcgen05 (fp32 accumulate)"},
            "plain": "fp32 CUDA cores, readout and >=2 contraction",
            "l2": "inputs and tables larger than L2 (126 MB): every step streams new showers",
            "parallelism": "replicas"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while it is open."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        # nvidia-smi takes a moment to start: wait for its first sample (taken
        # before the timed region, not kept) so that sampling runs throughout
        import select
        ready, _, _ = select.select([self.proc.stdout], [], [], 10.0)
        if ready:
            self.proc.stdout.readline()
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons),
                "window": "whole served, end-to-end and latency runs"}


# ------------------------------------------------------------------ CPU arm
def oracle_route(threads):
    from oracle.shower import Route
    return Route(np.load(TABLES / "route_c2.npz"), np.load(TABLES / "ge2_fold_384om_2-450m.npz"),
                 np.load(TABLES / "near_c2.npz"), order0_gauss=8, threads=threads)


ORACLE_SAMPLE = ("float64 CPU restatement of the reference's ShowerTransport route (oracle/: "
                 "order 1 and the >=2 contraction in C, sources in NumPy, first-entry order 0 "
                 "at Gauss order 8), the OM-parallel stages on one thread per host core")


def time_cpu_sample(pool, budget_s=20.0):
    """Showers of the stream, in order, through the CPU oracle until ``budget_s``
    of wall time has passed (at least one): (showers, seconds, cores)."""
    cores = os.cpu_count() or 1
    route = oracle_route(cores)
    done, t0 = 0, time.perf_counter()
    for el in pool:
        route(el)
        done += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    return done, time.perf_counter() - t0, cores


def reference_arm(args, rank):
    """The CPU restatement of the reference route on the host cores, one shower
    of the stream per step (no JIT: warm-up steps run the first showers)."""
    if rank != 0:
        return
    centroid = np.load(TABLES / "route_c2.npz")["positions_m"].mean(axis=0)
    pool = shower_pool(centroid, max(POOL, args.warmup + args.steps))
    cores = os.cpu_count() or 1
    route = oracle_route(cores)
    for k in range(args.warmup):
        route(pool[k])
    times = []
    for k in range(args.warmup, args.warmup + args.steps):
        t0 = time.perf_counter()
        route(pool[k])
        times.append(time.perf_counter() - t0)
    total = float(np.sum(times))
    value = args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "showers/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_json(pool[:POOL], args.steps),
            "cpu_baseline": {"value": value, "unit": "showers/s", "cores": cores, "kind": "port",
                             "sample": f"one shower of the stream per step: showers "
                                       f"{args.warmup}..{args.warmup + args.steps - 1} of the "
                                       f"seed-21 stream; {ORACLE_SAMPLE}"},
            "e2e": {"value": value, "unit": "showers/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ device arm
def response_bytes(r):
    return int(r.components_pe.nbytes + r.charge_components_pe.nbytes + r.spectrum_ge2_pe.nbytes
               + r.time_origin_ns.nbytes + r.active.nbytes)


def element_bytes(el):
    return int(sum(np.asarray(el[k]).nbytes for k in ("start_m", "direction", "length_m",
                                                      "coefficient0", "coefficient2", "beta",
                                                      "start_ns", "end_ns")))


def served_region(server, sources, stream):
    """Queue every source, wait for all: (ms on the device clock, results)."""
    import torch
    e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
    torch.cuda.synchronize()
    e0.record(stream)
    for s in sources:
        server.submit(s)
    done = server.drain(len(sources), timeout=1800)
    torch.cuda.synchronize()
    e1.record(stream)
    e1.synchronize()
    errors = [r.error for r in done if r.error is not None]
    if errors:
        raise errors[0]
    return e0.elapsed_time(e1), done


def shower_section(args, dev, world):
    import torch
    from lighthit_b200 import _lib
    from lighthit_b200.order0 import ResidentElements
    from lighthit_b200.serve_shower import ShowerServer
    from lighthit_b200.shower import ShowerSettings, ShowerTables, ShowerTransport
    stream = torch.cuda.current_stream(dev)
    plain = ShowerTransport(ShowerTables.synthetic(
        "c2", device=dev, settings=ShowerSettings(readout_mode="fp32", contraction_mode="fp32")))
    pool = shower_pool(plain.tables.positions.mean(axis=0))
    resident = [ResidentElements(el, dev) for el in pool]
    server = ShowerServer(lambda: ShowerTransport(ShowerTables.synthetic("c2", device=dev)),
                          workers=WORKERS, max_batch=MAX_BATCH)
    steps, warmup = args.steps, max(args.warmup, 3)
    try:
        # every worker's workspaces sized for the pool's two largest showers (on
        # each of its side-stream lanes), so no step allocates device memory
        largest = sorted(resident, key=lambda e: len(e["length_m"]))[-2:]
        server.prime(largest * server.routes[0].n_lanes)
        # warm-up: caching allocators filled, every kernel loaded
        served_region(server, [s for k in range(warmup) for s in step_showers(resident, k)],
                      stream)
        if world > 1:
            torch.distributed.barrier()
        timed = [s for k in range(steps) for s in step_showers(resident, k)]
        with ClockSampler(dev.index or 0) as clocks:
            _lib.kernel_timing(True)
            served_ms, _ = served_region(server, timed, stream)
            kernels = _lib.kernel_times()
            units = _lib.kernel_units()
            _lib.kernel_timing(False)
            if world > 1:
                torch.distributed.barrier()
            served_ms = max_over_ranks(served_ms, dev)
            # end to end: host element arrays in, every response field read back
            e2e_steps = max(1, min(steps, 8))
            host = [s for k in range(e2e_steps) for s in step_showers(pool, k)]
            e2e_ms, done = served_region(server, host, stream)
            e2e_ms = max_over_ranks(e2e_ms, dev)
            h2d = sum(element_bytes(s) for s in host) / e2e_steps
            d2h = sum(response_bytes(r.result) for r in done) / e2e_steps
            served_rate = job_rate(len(timed), world, served_ms)
            # latency under Poisson arrivals at half the served rate
            rng = np.random.default_rng(22)
            lat_showers = [s for k in range(4) for s in step_showers(resident, k)]
            arrivals = np.cumsum(rng.exponential(1.0 / (0.5 * served_rate / world),
                                                 size=len(lat_showers)))
            start = time.perf_counter()
            for k, el in enumerate(lat_showers):
                wait = start + arrivals[k] - time.perf_counter()
                if wait > 0:
                    time.sleep(wait)
                server.submit(el, arrival=start + arrivals[k])
            lat = np.array([r.latency for r in server.drain(len(lat_showers), timeout=1800)]) * 1e3
        # plain FP32 path: one shower per call on the same showers
        plain_showers = step_showers(resident, 0) + step_showers(resident, 1)
        for el in plain_showers[:3]:
            plain(el)
        p0, p1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
        torch.cuda.synchronize()
        p0.record(stream)
        for el in plain_showers:
            plain(el)
        torch.cuda.synchronize()
        p1.record(stream)
        p1.synchronize()
        plain_rate = len(plain_showers) / (p0.elapsed_time(p1) / 1e3)
        # launches of this library's kernels per step, counted in one untimed step
        launches = count_launches(server, step_showers(resident, 0))
    finally:
        server.close()
    return dict(pool=pool, served_ms=served_ms, served_rate=served_rate, steps=steps,
                warmup=warmup, e2e_ms=e2e_ms, e2e_steps=e2e_steps, e2e_rate=job_rate(
                    len(host), world, e2e_ms), h2d=h2d, d2h=d2h, lat=lat, clocks=clocks.summary(),
                kernels=kernels, units=units, plain_rate=plain_rate, plain_n=len(plain_showers),
                launches_per_step=launches)


def count_launches(server, sources):
    """Kernels of this library launched for ``sources`` (one profiled, untimed run)."""
    import torch
    from torch.profiler import ProfilerActivity, profile
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for s in sources:
            server.submit(s)
        server.drain(len(sources), timeout=1800)
        torch.cuda.synchronize()
    return sum(1 for e in prof.events() if e.device_type.name == "CUDA"
               and e.name.startswith("lh::"))


def shower_roofline(kernels, hbm_peak, peak_source):
    """Roofline of the order-1 group stage (``o1_group_kernel``), the row's unit
    being one (OM, pencil) evaluation that reads one float64 pencil record
    (``PENCIL_BYTES``): achieved = evaluations per launch x record bytes over the
    launch's average CUDA-event duration, both measured in the timed region."""
    group = kernels.get("o1_group_kernel")
    if not group or not group["units"]:
        return None
    per_launch = group["units"] / group["launches"]
    achieved = per_launch * PENCIL_BYTES / (group["avg_ms"] / 1e3) / 1e9
    traffic = (None if O1_GROUP_TRAFFIC_PER_ITEM is None
               else O1_GROUP_TRAFFIC_PER_ITEM * per_launch)
    return {"kernel": "o1_group_kernel", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
            "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": traffic,
            "peak_source": peak_source, "algorithmic_bytes_per_unit": PENCIL_BYTES,
            "unit_of_work": "(OM, pencil) evaluation", "units_per_launch": per_launch,
            "avg_launch_ms": group["avg_ms"], "launches": group["launches"],
            "note": "the pencil table (a few MB) stays in L2, so DRAM traffic is far below "
                    "the algorithmic bytes: the kernel is bound by float64 issue and latency "
                    "(see profiles/), not by HBM"}


def contraction_roofline(kernels, tensor_peak, peak_source):
    """The tensor-core >=2 contraction against the BF16 tensor peak, in the GEMM
    convention of the scope table: 2 x rows x K x N flops with rows = in-window
    (OM, point) pairs x 39 source channels, K = 6 pairs x 4 powers, N = 2 x 65
    frequencies x 3 bands, per split-BF16 product set counted once."""
    ge2 = kernels.get("ge2_tc_kernel")
    if not ge2 or not ge2["units"]:
        return None
    flops = ge2["units"] * 39 * 2 * 24 * 390 / ge2["launches"]
    achieved = flops / (ge2["avg_ms"] / 1e3) / 1e12
    return {"kernel": "ge2_tc_kernel", "bound": "tensor", "achieved": achieved,
            "peak": tensor_peak, "unit": "TFLOP/s", "frac": achieved / tensor_peak,
            "peak_source": peak_source, "pairs_per_launch": ge2["units"] / ge2["launches"],
            "flops_per_launch": flops, "avg_launch_ms": ge2["avg_ms"],
            "note": "the contraction's K is 24 and each output needs a complex channel "
                    "product in the epilogue, so the CUDA-core epilogue and the operand "
                    "loads, not the MMAs, bound it"}


def flash_section(args, dev):
    """Config 1 (4096 isotropic 450 nm flashes, uneven batches) as an extra key."""
    import torch
    from lighthit_b200.flash import FlashTable, FlashTransport
    from lighthit_b200.model import KernelConfig, synthetic_detector
    from lighthit_b200.workloads import flash_batch_sizes, flash_positions
    det = synthetic_detector()
    cfg = KernelConfig(omega_per_ns=np.linspace(0, 1.2, 65),
                       readout_omega_per_ns=np.linspace(0, 1.2, 321),
                       relative_time_edges_ns=np.arange(-60.0, 745.0, 5.0),
                       radial_range_m=(2.0, 250.0), threshold_pe=0.01)
    pos_np = flash_positions(N_FLASH, det.positions_m.mean(axis=0), seed=11,
                             om_positions=det.positions_m)
    table = FlashTable.load(FLASH_TABLE)
    served = FlashTransport(det, cfg, table, device=dev, mode="split-bf16")
    plain = FlashTransport(det, cfg, table, device=dev, mode="fp32")
    pos = torch.tensor(pos_np, dtype=torch.float64, device=dev)
    ph = torch.full((N_FLASH,), 1e10, dtype=torch.float64, device=dev)
    tt = torch.zeros(N_FLASH, dtype=torch.float64, device=dev)
    out = served.allocate(N_FLASH)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(3):
        served.launch(pos, ph, tt, out, stream=stream)
    torch.cuda.synchronize(dev)
    served.raise_for_status(out)
    n = max(3, min(args.steps, 50))
    ms = []
    for k in range(n):
        flush.fill_(k & 0xFF)
        e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
        e0.record(stream)
        served.launch(pos, ph, tt, out, stream=stream)
        e1.record(stream)
        ms.append((e0, e1))
    torch.cuda.synchronize(dev)
    step_ms = np.array([a.elapsed_time(b) for a, b in ms])
    per_pair = 65 * 3 * 8 + 3 * 160 * 4 + 3 * 8 + 8 + 1
    achieved = per_pair * 48 * N_FLASH / (step_ms.mean() / 1e3) / 1e9
    pout = plain.allocate(1)
    p0, p1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
    for i in range(4):
        plain.launch(pos[i:i + 1], ph[i:i + 1], tt[i:i + 1], pout, stream=stream)
    p0.record(stream)
    for i in range(256):
        plain.launch(pos[i:i + 1], ph[i:i + 1], tt[i:i + 1], pout, stream=stream)
    p1.record(stream)
    torch.cuda.synchronize(dev)
    return {"workload": "config 1: 4096 isotropic 450 nm flashes (1e10 photons, seed 11) on the "
                        "48-OM array, one fused launch", "value": N_FLASH / (step_ms.mean() / 1e3),
            "unit": "flashes/s", "ms_per_launch": float(step_ms.mean()), "launches": n,
            "plain_fp32": {"value": 256 / (p0.elapsed_time(p1) / 1e3), "unit": "flashes/s",
                           "launch": "one flash per launch"},
            "roofline": {"kernel": "flash_tc_kernel", "bound": "hbm", "achieved": achieved,
                         "unit": "GB/s", "algorithmic_bytes_per_pair": per_pair,
                         "pairs_per_launch": 48 * N_FLASH, "traffic": FLASH_TC_TRAFFIC},
            "l2": "flushed between launches"}


def kernel_case(args):
    """One stage-major batch of the first ``args.kernel_case`` showers of the
    stream through ``ShowerTransport.batch`` (after one untimed batch): the
    small case the ncu captures of the shower kernels run on. Prints the timed
    kernels of the second batch."""
    import torch
    from lighthit_b200 import _lib
    from lighthit_b200.shower import ShowerTables, ShowerTransport
    route = ShowerTransport(ShowerTables.synthetic("c2"))
    pool = shower_pool(route.tables.positions.mean(axis=0), args.kernel_case)
    route.batch(pool)
    torch.cuda.synchronize()
    _lib.kernel_timing(True)
    route.batch(pool)
    torch.cuda.synchronize()
    times = _lib.kernel_times()
    units = _lib.kernel_units()
    _lib.kernel_timing(False)
    print(json.dumps({"case": f"first {len(pool)} showers of the config-2 stream, one batch",
                      "kernels": {k: {"launches": n, "total_ms": ms, "units": units.get(k)}
                                  for k, (n, ms) in times.items()}}), flush=True)


def ours(args, rank, world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (
        ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_source = ("MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks
                   else "fallback 6650 GB/s (no MEASURED_PEAKS.json)")
    s = shower_section(args, dev, world)
    flash = None if args.no_flash else flash_section(args, dev)
    if flash is not None:
        flash["roofline"].update(peak=hbm_peak, frac=flash["roofline"]["achieved"] / hbm_peak,
                                 peak_source=peak_source)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        done, secs, cores = time_cpu_sample(s["pool"])
        cpu = {"value": done / secs, "unit": "showers/s", "cores": cores, "kind": "port",
               "sample": f"the first {done} showers of the stream ({secs:.1f} s); {ORACLE_SAMPLE}"}
    if rank != 0:
        return
    kernels = {k: {"launches": n, "total_ms": ms, "avg_ms": ms / n, "units": s["units"].get(k)}
               for k, (n, ms) in s["kernels"].items()}
    top = max(kernels.items(), key=lambda kv: kv[1]["total_ms"])[0] if kernels else None
    roof = shower_roofline(kernels, hbm_peak, peak_source)
    tensor_peak = float(peaks.get("bf16_tflops", 1590.0))
    contraction = contraction_roofline(
        kernels, tensor_peak, "MEASURED_PEAKS.json bf16_tflops (measured)"
        if "bf16_tflops" in peaks else "fallback 1590 TFLOP/s (no MEASURED_PEAKS.json)")
    line = {
        "metric": METRIC, "value": s["served_rate"], "unit": "showers/s", "n_gpus": world,
        "steps": s["steps"], "warmup": s["warmup"],
        "ms_per_step": s["served_ms"] / s["steps"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 geometry and clocks, f64 order 1, f32 order 0, split-bf16 >=2 "
                 "contraction and readout on the tensor cores (f32 accumulate)",
        "data": "synthetic", "config": config_json(s["pool"], s["steps"]),
        "latency": {"p50_ms": float(np.percentile(s["lat"], 50)),
                    "p99_ms": float(np.percentile(s["lat"], 99)), "requests": len(s["lat"]),
                    "offered_showers_per_s": 0.5 * s["served_rate"] / world,
                    "definition": "Poisson arrival to the response on the host, serving loop"},
        "plain_fp32": {"value": s["plain_rate"], "unit": "showers/s", "showers": s["plain_n"],
                       "launch": "ShowerTransport per shower on one stream, fp32 readout"},
        "served_over_plain": s["served_rate"] / world / s["plain_rate"],
        "roofline": roof, "contraction_roofline": contraction, "kernel_times": kernels,
        "top_kernel": top,
        "cpu_baseline": cpu,
        "e2e": {"value": s["e2e_rate"], "unit": "showers/s",
                "h2d_bytes_per_step": int(s["h2d"]), "d2h_bytes_per_step": int(s["d2h"]),
                "steps": s["e2e_steps"],
                "path": "ShowerServer.submit of host element arrays -> responses on the host "
                        "(charge, bins, spectrum, clocks, active)"},
        "gpu_launches": int(s["launches_per_step"] * s["steps"]),
        "gpu_launches_method": "kernels of liblh_b200 in one profiled untimed step x steps",
        "flash_stream": flash,
        "clocks": s["clocks"],
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-flash", action="store_true", help="skip the flash-stream section")
    ap.add_argument("--kernel-case", type=int, default=0, metavar="N",
                    help="run only one batch of N showers (the case of the ncu captures)")
    args = ap.parse_args()
    if args.kernel_case:
        kernel_case(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
