#!/usr/bin/env python
"""Served calibration-flash stream on the B200 (one JSON line on rank 0).

Workload: 4096 monochromatic 450 nm isotropic flashes of 1e10 photons, uniform
in a cylinder (r 60 m, h 300 m) around the centroid of the 48-OM synthetic
array (seed 11), served in uneven batches of 1-256 flashes (seed 12); orders
0, 1 and >=2 from the multipole table, 65 RTE frequencies, 321-node readout,
160 bins of 5 ns. A step is one pass over the whole stream.

* ``value``: flashes/s of the served mixed-precision path (fused tcgen05
  kernel, split-BF16 readout, fp32 accumulate), inputs resident in HBM,
  CUDA-event timed, L2 flushed between steps.
* ``plain_fp32``: the plain FP32 GPU path launched once per flash.
* ``e2e``: the same stream through the public batch API from pinned host
  buffers, every response field copied back to the host each step.
* ``cpu_baseline``: the CPU oracle on a bounded sample on this host.

``--impl reference`` times the reference algorithm on the host CPU (the oracle
port, all cores) on the same workload and prints the same line.
``--gpus N`` under torchrun runs N independent replicas (weak scaling).
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
TABLE = ROOT / "lighthit_b200" / "tables" / "flash_450nm_2-250m.npz"
N_FLASH = 4096
# DRAM bytes (read + write) of one 4096-flash flash_tc_kernel launch, measured with
# ncu on a B200 (profiles/flash_tc_kernel_4096flashes.txt).
FLASH_TC_TRAFFIC = 636_147_456


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


def workload():
    from lighthit_b200.model import KernelConfig, synthetic_detector
    from lighthit_b200.workloads import flash_batch_sizes, flash_positions
    det = synthetic_detector()
    cfg = KernelConfig(omega_per_ns=np.linspace(0, 1.2, 65),
                       readout_omega_per_ns=np.linspace(0, 1.2, 321),
                       relative_time_edges_ns=np.arange(-60.0, 745.0, 5.0),
                       radial_range_m=(2.0, 250.0), threshold_pe=0.01)
    pos = flash_positions(N_FLASH, det.positions_m.mean(axis=0), seed=11,
                          om_positions=det.positions_m)
    sizes = flash_batch_sizes(N_FLASH, seed=12)
    return det, cfg, pos, sizes


def config_json(sizes):
    return {"workload": "config 1: 4096 isotropic 450 nm flashes (1e10 photons, seed 11) on "
                        "the 48-OM synthetic array, served in uneven batches of 1-256",
            "flashes_per_step": N_FLASH, "batches_per_step": len(sizes),
            "n_om": 48, "omega_nodes": 65, "readout_nodes": 321, "bins": 160,
            "table": "2-250 m, 48 radial nodes, degree 8", "l2": "flushed between steps",
            "parallelism": "replicas"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
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
                "samples": len(sm), "reasons": sorted(reasons)}


def time_cpu_oracle(pos, det, cfg, sample):
    """Oracle (float64 NumPy restatement of the reference) on ``sample`` flashes."""
    from lighthit_b200.model import acceptance_coefficients
    table = dict(np.load(TABLE))
    alpha = acceptance_coefficients(det.angular_acceptance, int(table["degree"]))
    job = dict(table=table, det=dict(positions_m=det.positions_m, orientations=det.orientations,
                                     area_m2=np.full(len(det), np.pi * 0.2 ** 2), alpha=alpha,
                                     spectral_weight=float(det.spectral_weight(450.0))),
               cfg=dict(omega_per_ns=cfg.omega_per_ns, readout_omega_per_ns=cfg.readout_omega_per_ns,
                        edges_ns=cfg.relative_time_edges_ns, threshold_pe=cfg.threshold_pe,
                        radial_range_m=cfg.radial_range_m))
    _oracle_one((job, pos[0]))  # build the table spline once, as the reference caches it
    t0 = time.perf_counter()
    for i in range(sample):
        _oracle_one((job, pos[i]))
    return time.perf_counter() - t0


_JOB = None


def _oracle_init(job):
    global _JOB
    _JOB = job


def _oracle_one(arg):
    job, p = arg if isinstance(arg, tuple) else (_JOB, arg)
    from oracle.flash import transport_flash
    det = dict(job["det"], acceptance=lambda x: .45 + .45 * np.asarray(x) + .10 * np.asarray(x) ** 2)
    return transport_flash(job["table"], det, dict(position_m=p, photons=1e10, time_ns=0.0),
                           job["cfg"])["charge_components_pe"].sum()


def reference_arm(args, rank):
    if rank != 0:
        return
    import multiprocessing as mp
    from lighthit_b200.model import acceptance_coefficients
    det, cfg, pos, sizes = workload()
    cores = os.cpu_count() or 1
    sample = max(cores * 8, 32)
    table = dict(np.load(TABLE))
    alpha = acceptance_coefficients(det.angular_acceptance, int(table["degree"]))
    job = dict(table=table, det=dict(positions_m=det.positions_m, orientations=det.orientations,
                                     area_m2=np.full(len(det), np.pi * 0.2 ** 2), alpha=alpha,
                                     spectral_weight=float(det.spectral_weight(450.0))),
               cfg=dict(omega_per_ns=cfg.omega_per_ns, readout_omega_per_ns=cfg.readout_omega_per_ns,
                        edges_ns=cfg.relative_time_edges_ns, threshold_pe=cfg.threshold_pe,
                        radial_range_m=cfg.radial_range_m))
    times = []
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"  # one thread per worker process, one worker per core
    with mp.get_context("spawn").Pool(cores, initializer=_oracle_init, initargs=(job,)) as pool:
        for k in range(args.warmup + args.steps):
            chunk = [pos[(k * sample + i) % N_FLASH] for i in range(sample)]
            t0 = time.perf_counter()
            pool.map(_oracle_one, chunk, chunksize=max(1, sample // cores))
            if k >= args.warmup:
                times.append(time.perf_counter() - t0)
    per_flash = float(np.median(times)) / sample
    value = 1.0 / per_flash
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "flashes/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": per_flash * N_FLASH * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_json(sizes),
            "cpu_baseline": {"value": value, "unit": "flashes/s", "cores": cores, "kind": "port",
                             "sample": f"{sample} flashes of the 4096-flash stream per step, "
                                       f"float64 oracle restatement of the reference route"},
            "e2e": {"value": value, "unit": "flashes/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


N_SHOWER = 96


def shower_stream_section(dev, steps, workers=3, max_batch=8):
    """Config 2: the served shower stream at 384 OMs through the device route.

    ``plain_fp32``: one shower after another on one stream, fp32 readout (the
    per-event path). ``served``: the serving loop (continuous batching of up to
    ``max_batch`` queued showers per stage-major batch, ``workers`` worker
    streams), split-BF16 readout. Wall time with the device synchronised on both sides
    (several streams and host orchestration: the device clock of one stream
    does not cover the job).
    """
    import torch
    from lighthit_b200.serve_shower import ShowerServer
    from lighthit_b200.shower import ShowerSettings, ShowerTables, ShowerTransport
    from lighthit_b200.workloads import gaussian_shower, shower_stream
    plain = ShowerTransport(ShowerTables.synthetic("c2", device=dev,
                                                   settings=ShowerSettings(readout_mode="fp32")))
    centroid = plain.tables.positions.mean(axis=0)
    draws = shower_stream(N_SHOWER, centroid)
    showers = [gaussian_shower(d["position_m"], d["direction"],
                               charged_track_length_m=d["charged_track_length_m"],
                               elements=d["elements"], seed=d["seed"]) for d in draws]
    for el in showers[:3]:
        plain(el)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    reps = max(1, min(steps, 2))
    stage = {}
    for _ in range(reps):
        for el in showers:
            r = plain(el)
            for k, v in r.metadata["timings"].items():
                stage[k] = stage.get(k, 0.0) + v
    torch.cuda.synchronize(dev)
    plain_s = (time.perf_counter() - t0) / reps
    server = ShowerServer(lambda: ShowerTransport(ShowerTables.synthetic("c2", device=dev)),
                          workers=workers, max_batch=max_batch)
    for el in showers[:workers]:
        server.submit(el)
    server.drain(workers)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(reps):
        for el in showers:
            server.submit(el)
        done = server.drain(len(showers))
        assert all(r.error is None for r in done), [r.error for r in done if r.error][:1]
    torch.cuda.synchronize(dev)
    served_s = (time.perf_counter() - t0) / reps
    served_rate = len(showers) / served_s
    # latency under Poisson arrivals at half the served rate
    rng = np.random.default_rng(22)
    arrivals = np.cumsum(rng.exponential(1.0 / (0.5 * served_rate), size=len(showers)))
    start = time.perf_counter()
    for k, el in enumerate(showers):
        wait = start + arrivals[k] - time.perf_counter()
        if wait > 0:
            time.sleep(wait)
        server.submit(el, arrival=start + arrivals[k])
    lat = np.array([r.latency for r in server.drain(len(showers))]) * 1e3
    server.close()
    sizes = [d["elements"] for d in draws]
    return {"workload": f"config 2: {N_SHOWER} Gaussian showers of the seed-21 stream "
                        "(500-50000 elements log-uniform, 0.15 m per element, vertices in a "
                        "200 m x 600 m cylinder, isotropic) on the 384-OM array, tables 2-450 m",
            "value": served_rate, "unit": "showers/s", "served_workers": workers,
            "max_batch": max_batch,
            "plain_fp32": {"value": len(showers) / plain_s, "unit": "showers/s",
                           "launch": "the device route per shower on one stream, fp32 readout"},
            "served_over_plain": served_rate * plain_s / len(showers),
            "latency": {"p50_ms": float(np.percentile(lat, 50)),
                        "p99_ms": float(np.percentile(lat, 99)),
                        "offered_showers_per_s": 0.5 * served_rate, "requests": len(lat)},
            "elements_per_shower": {"min": int(min(sizes)), "median": int(np.median(sizes)),
                                    "max": int(max(sizes))},
            "plain_stage_ms_per_shower": {k: 1e3 * v / (reps * len(showers))
                                          for k, v in sorted(stage.items(), key=lambda x: -x[1])},
            "timing": "wall clock, device synchronised before and after"}


def _events(torch, n):
    return [torch.cuda.Event(enable_timing=True) for _ in range(n)]


def ours(args, rank, world, local_rank):
    import torch
    from lighthit_b200.flash import FlashTable, FlashTransport
    from lighthit_b200.serve import FlashServer, ServeConfig, autotune, flash_bytes
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    det, cfg, pos_np, sizes = workload()
    table = FlashTable.load(TABLE)
    served = FlashTransport(det, cfg, table, device=dev, mode="split-bf16")
    plain = FlashTransport(det, cfg, table, device=dev, mode="fp32")
    F = N_FLASH
    threads = autotune(served, F, cache=str(ROOT / "_work" / "autotune.json")
                       if (ROOT / "_work").exists() else None)
    pos = torch.tensor(pos_np, dtype=torch.float64, device=dev)
    ph = torch.full((F,), 1e10, dtype=torch.float64, device=dev)
    tt = torch.zeros(F, dtype=torch.float64, device=dev)
    out = served.allocate(F)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    bounds = np.concatenate([[0], np.cumsum(sizes)])
    requests = [(int(a), int(b)) for a, b in zip(bounds[:-1], bounds[1:])]

    # Served launches: the loop coalesces every queued request into one launch
    # per free slot, so with the whole stream queued a step is one fused launch.
    def coalesced(ev=None):
        if ev is not None:
            ev[0].record(stream)
        served.launch(pos, ph, tt, out, stream=stream, block_threads=threads)
        if ev is not None:
            ev[1].record(stream)

    for _ in range(max(args.warmup, 3)):
        coalesced()
    torch.cuda.synchronize(dev)
    served.raise_for_status(out)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    ev = [_events(torch, 2) for _ in range(args.steps)]
    with ClockSampler(local_rank) as clocks:
        for k in range(args.steps):
            flush.fill_(k & 0xFF)  # write > L2 between timed steps (outside the events)
            coalesced(ev[k])
        torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    step_ms = np.array([a.elapsed_time(b) for a, b in ev])
    total_ms = float(step_ms.sum())
    total_ms = max_over_ranks(total_ms, dev)
    value = job_rate(F * args.steps, world, total_ms)

    # roofline of the fused kernel: algorithmic bytes = outputs written per (flash, OM)
    per_pair = 65 * 3 * 8 + 3 * 160 * 4 + 3 * 8 + 8 + 1
    achieved = per_pair * 48 * F * args.steps / (step_ms.sum() / 1e3) / 1e9
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (
        ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))

    # one launch per request (no coalescing), same kernel
    views = []
    for a, b in requests:
        v = {k: t[a:b] for k, t in out.items() if k != "status"}
        v["status"] = torch.zeros(4, dtype=torch.int32, device=dev)
        views.append(v)
    pr_steps = min(args.steps, 20)
    r0, r1 = _events(torch, 2)
    r0.record(stream)
    for _ in range(pr_steps):
        for i, (a, b) in enumerate(requests):
            served.launch(pos[a:b], ph[a:b], tt[a:b], views[i], stream=stream, block_threads=threads)
    r1.record(stream)
    torch.cuda.synchronize(dev)
    per_request_value = F * pr_steps / (r0.elapsed_time(r1) / 1e3)

    # plain FP32 path, one launch per flash
    n_plain = min(512, F)
    pout = plain.allocate(1)
    for i in range(8):
        plain.launch(pos[i:i + 1], ph[i:i + 1], tt[i:i + 1], pout, stream=stream)
    torch.cuda.synchronize(dev)
    p0, p1 = _events(torch, 2)
    p0.record(stream)
    for i in range(n_plain):
        plain.launch(pos[i:i + 1], ph[i:i + 1], tt[i:i + 1], pout, stream=stream)
    p1.record(stream)
    torch.cuda.synchronize(dev)
    plain_value = n_plain / (p0.elapsed_time(p1) / 1e3)

    # end to end: the serving loop (public API) from host arrays to host results,
    # every response field copied back; all requests queued at once
    cap = 2048
    srv = FlashServer(served, ServeConfig(hbm_budget_bytes=2 * cap * flash_bytes(48, 65, 160),
                                          slots=2, max_flashes_per_launch=cap,
                                          block_threads=threads))

    def serve_all():
        """One step: every request submitted, served and handed back; the client
        then drops the results, so their pinned buffers return to the host pool."""
        for a, b in requests:
            srv.submit(pos_np[a:b], 1e10)
        srv.poll()
        done = srv.drain()
        served_flashes = sum(len(r.positions) for r in done)
        assert served_flashes == F and all(r.error is None for r in done)
        shape = done[0].result["charge"].shape
        srv.completed.clear()
        return shape

    first_shape = serve_all()
    assert first_shape == (requests[0][1] - requests[0][0], 48, 3)
    serve_all()
    e2e_steps = min(args.steps, 20)
    e0, e1 = _events(torch, 2)
    torch.cuda.synchronize(dev)
    w0 = time.perf_counter()
    e0.record(stream)
    for _ in range(e2e_steps):
        serve_all()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - w0
    e2e_ms = e0.elapsed_time(e1)
    e2e_ms = max_over_ranks(e2e_ms, dev)
    e2e_value = job_rate(F * e2e_steps, world, e2e_ms)
    h2d = F * (3 * 8 + 8 + 8)
    d2h = F * 48 * per_pair

    # latency under Poisson arrivals at half the end-to-end capacity
    srv.completed.clear()
    offered = 0.5 * F * e2e_steps / wall
    rng = np.random.default_rng(13)
    mean_req = F / len(requests)
    arrivals = np.cumsum(rng.exponential(mean_req / offered, size=len(requests) * 3))
    order = [requests[i % len(requests)] for i in range(len(arrivals))]
    t_start = time.perf_counter()
    nxt = 0
    latencies = []
    while nxt < len(arrivals) or srv.queue or srv.busy:
        now = time.perf_counter() - t_start
        while nxt < len(arrivals) and arrivals[nxt] <= now:
            a, b = order[nxt]
            srv.submit(pos_np[a:b], 1e10, arrival=t_start + arrivals[nxt])
            nxt += 1
        srv.poll()
        latencies += [r.latency for r in srv.completed]
        srv.completed.clear()  # the client takes each result as it completes
    lat_ms = np.array(latencies) * 1e3

    showers = None
    if not args.no_showers:
        showers = shower_stream_section(dev, args.steps)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sample = 128
        secs = time_cpu_oracle(pos_np, det, cfg, sample)
        cpu = {"value": sample / secs, "unit": "flashes/s", "cores": 1, "kind": "port",
               "sample": f"first {sample} flashes of the stream, float64 oracle restatement "
                         "of the reference route, one process"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "flashes/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 spectrum, split-bf16 readout (f32 accumulate), f64 clocks",
            "data": "synthetic", "config": config_json(sizes),
            "latency": {"p50_ms": float(np.percentile(lat_ms, 50)),
                        "p99_ms": float(np.percentile(lat_ms, 99)),
                        "offered_flashes_per_s": offered, "requests": len(lat_ms),
                        "definition": "request arrival (Poisson, uneven 1-256 flash requests) to "
                                      "every response field on the host, serving loop, 2 slots"},
            "served_per_request_launch": {"value": per_request_value, "unit": "flashes/s",
                                          "launches_per_step": len(requests)},
            "plain_fp32": {"value": plain_value, "unit": "flashes/s",
                           "launch": "one flash per launch (2 kernels), fp32 CUDA-core readout",
                           "sample": n_plain},
            "served_over_plain": value / world / plain_value,
            "roofline": {"kernel": "flash_tc_kernel", "bound": "hbm", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)",
                         "algorithmic_bytes_per_pair": per_pair, "pairs_per_launch": 48 * F,
                         "block_threads": threads, "traffic": FLASH_TC_TRAFFIC,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one "
                                           "4096-flash launch (profiles/flash_tc_kernel_4096flashes.txt)"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "flashes/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "wall_s": wall, "steps": e2e_steps,
                    "path": "FlashServer (serving loop): pinned staging, graph replay, D2H of "
                            "every response field"},
            "shower_stream": showers,
            "gpu_launches": args.steps,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-showers", action="store_true", help="skip the shower-stream section")
    args = ap.parse_args()
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
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
