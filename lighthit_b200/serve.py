"""Persistent request loop for calibration flashes (continuous batching).

Requests are flash batches of uneven size submitted from the host as they
arrive. The loop keeps a few launch *slots*; each slot owns pinned host
staging, device inputs, device outputs and pinned host result buffers, sized
by the HBM budget. ``poll()``:

1. finishes every slot whose launch has completed: the results of each request
   in it are handed back (host arrays, with the reference's error for any flash
   that raised on the device) and the slot is free again;
2. admits queued requests into free slots, first come first served, as many as
   fit the slot's capacity (a request larger than a slot is split), stages
   their inputs, replays the slot's captured CUDA graph (input copy, status
   reset, fused kernel reading the flash count from device memory) and queues
   the copy of exactly the filled part of the outputs back to the host.

Slots run on their own streams, so one launch computes while the host stages
the next and drains the previous; requests that arrive while others are on the
GPU join the next launch as soon as a slot frees. The fused kernel's CTA size
is picked by :func:`autotune` and cached on disk.

The device-specific work sits behind a small backend interface, so the queue,
admission and splitting logic run unchanged against a host fake in tests.
"""
from __future__ import annotations

import json
import os
import time
from collections import deque
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _lib

__all__ = ["ServeConfig", "FlashRequest", "FlashServer", "CudaFlashBackend", "autotune",
           "flash_bytes"]

RESULT_KEYS = ("spectrum", "components", "charge", "origin", "active")


@dataclass(frozen=True)
class ServeConfig:
    """Serving settings: HBM budget for the slots, slot count, launch cap, graphs, tuning."""
    hbm_budget_bytes: int = 8 << 30
    slots: int = 2
    max_flashes_per_launch: int = 4096
    use_graphs: bool = True
    autotune_cache: str | None = None
    block_threads: int | None = None  # None: autotune (or 512 without a cache)


def flash_bytes(n_om, n_omega, n_bins):
    """Device bytes one flash occupies in a slot (inputs + every output field)."""
    return 5 * 8 + n_om * (n_omega * 3 * 8 + 3 * n_bins * 4 + 3 * 8 + 8 + 1)


@dataclass
class FlashRequest:
    rid: int
    positions: np.ndarray
    photons: np.ndarray
    time_ns: np.ndarray
    arrival: float
    done: float | None = None
    result: dict | None = None
    error: str | None = None
    _parts: list = field(default_factory=list)
    _pending: int = 0

    @property
    def latency(self):
        return None if self.done is None else self.done - self.arrival


class FlashServer:
    """Continuous-batching front end over a backend (default: the CUDA backend)."""

    def __init__(self, transport=None, config: ServeConfig | None = None, *, backend=None):
        self.config = config or ServeConfig()
        self.backend = backend or CudaFlashBackend(transport, self.config)
        cap = self.backend.capacity
        if cap < 1:
            raise MemoryError("the HBM budget does not hold one flash per slot")
        self.capacity = cap
        self.queue: deque = deque()      # (request, start, count) chunks awaiting a slot
        self.free = list(range(self.backend.n_slots))
        self.busy: dict = {}             # slot -> [(request, start, count, offset)]
        self.launches = 0
        self.completed: list = []
        self._next = 0

    def submit(self, positions, photons, time_ns=None, *, arrival=None):
        positions = np.asarray(positions, float).reshape(-1, 3)
        n = len(positions)
        photons = np.broadcast_to(np.asarray(photons, float), (n,)).copy()
        time_ns = (np.zeros(n) if time_ns is None
                   else np.broadcast_to(np.asarray(time_ns, float), (n,)).copy())
        req = FlashRequest(self._next, positions, photons, time_ns,
                           time.perf_counter() if arrival is None else arrival)
        self._next += 1
        for start in range(0, n, self.capacity):
            count = min(self.capacity, n - start)
            self.queue.append((req, start, count))
            req._pending += 1
        if n == 0:
            req.done, req.result = req.arrival, {}
            self.completed.append(req)
        return req

    def poll(self):
        """Finish completed slots, then fill free slots. Returns requests finished now."""
        finished = []
        for slot in list(self.busy):
            if self.backend.ready(slot):
                finished += self._finish(slot)
        while self.queue and self.free:
            slot = self.free.pop(0)
            items, used = [], 0
            while self.queue and used + self.queue[0][2] <= self.capacity:
                req, start, count = self.queue.popleft()
                items.append((req, start, count, used))
                used += count
            self.backend.stage(slot, [(r.positions[s:s + c], r.photons[s:s + c],
                                       r.time_ns[s:s + c], off) for r, s, c, off in items], used)
            self.backend.launch(slot, used, [(off, c) for _, _, c, off in items])
            self.busy[slot] = items
            self.launches += 1
        return finished

    def _finish(self, slot):
        items = self.busy.pop(slot)
        outs = self.backend.collect(slot)  # one dict of host arrays per admitted chunk
        self.free.append(slot)
        now = time.perf_counter()
        done = []
        for (req, start, count, off), part in zip(items, outs):
            req._parts.append((start, part))
            flags = part["active"] >> 1
            if np.any(flags) and req.error is None:
                bad = int(np.flatnonzero(np.any(flags, axis=1))[0]) + start
                req.error = ("isotropic point source cannot coincide with an OM centre"
                             if np.any(flags[bad - start] & 2) else
                             "OMs outside radial_range_m have an absorption-only estimate "
                             f"above threshold (flash {bad} of request {req.rid})")
            req._pending -= 1
            if req._pending == 0:
                parts = sorted(req._parts, key=lambda p: p[0])
                req.result = (dict(parts[0][1]) if len(parts) == 1 else
                              {k: np.concatenate([p[1][k] for p in parts]) for k in RESULT_KEYS})
                req.result["active"] = (req.result["active"] & 1).astype(bool)
                req._parts = []
                req.done = now
                done.append(req)
                self.completed.append(req)
        return done

    def drain(self, timeout_s=60.0):
        """Poll until every submitted request has finished."""
        t_end = time.perf_counter() + timeout_s
        while self.queue or self.busy:
            self.poll()
            if time.perf_counter() > t_end:
                raise TimeoutError("serving loop did not drain in time")
        return self.completed


# ---------------------------------------------------------------------- CUDA backend
class CudaFlashBackend:
    """Slots on CUDA streams with captured graphs around the fused flash kernel."""

    def __init__(self, transport, config: ServeConfig):
        import torch
        self.torch = torch
        self.t = transport
        self.config = config
        dev = transport.device
        per = flash_bytes(transport.n_om, transport.n_omega, transport.n_bins)
        cap = int(min(config.max_flashes_per_launch,
                      config.hbm_budget_bytes // (max(config.slots, 1) * per)))
        self.capacity = cap
        self.n_slots = int(config.slots)
        self.block_threads = config.block_threads or autotune(
            transport, min(cap, 1024), cache=config.autotune_cache)
        self.slots = []
        for _ in range(self.n_slots):
            s = dict(stream=torch.cuda.Stream(dev), event=torch.cuda.Event())
            s["h_pos"] = torch.zeros((cap, 3), dtype=torch.float64).pin_memory()
            s["h_ph"] = torch.zeros(cap, dtype=torch.float64).pin_memory()
            s["h_t"] = torch.zeros(cap, dtype=torch.float64).pin_memory()
            s["h_n"] = torch.zeros(1, dtype=torch.int32).pin_memory()
            s["d_pos"] = torch.zeros((cap, 3), dtype=torch.float64, device=dev)
            s["d_ph"] = torch.zeros(cap, dtype=torch.float64, device=dev)
            s["d_t"] = torch.zeros(cap, dtype=torch.float64, device=dev)
            s["d_n"] = torch.zeros(1, dtype=torch.int32, device=dev)
            s["out"] = transport.allocate(cap)
            s["graph"] = None
            s["parts"] = None
            s["count"] = 0
            self.slots.append(s)
        for i in range(self.n_slots):
            self._capture(i)

    def _body(self, s):
        s["d_pos"].copy_(s["h_pos"], non_blocking=True)
        s["d_ph"].copy_(s["h_ph"], non_blocking=True)
        s["d_t"].copy_(s["h_t"], non_blocking=True)
        s["d_n"].copy_(s["h_n"], non_blocking=True)
        s["out"]["status"].zero_()
        self.t.launch(s["d_pos"], s["d_ph"], s["d_t"], s["out"], n_device=s["d_n"],
                      block_threads=self.block_threads)

    def _capture(self, i):
        torch = self.torch
        s = self.slots[i]
        with torch.cuda.stream(s["stream"]):
            s["h_n"][0] = 0
            self._body(s)  # warm-up outside the graph (attributes, lazy module load)
        s["stream"].synchronize()
        if self.config.use_graphs:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s["stream"]):
                self._body(s)
            s["graph"] = g

    def stage(self, slot, parts, used):
        s = self.slots[slot]
        for pos, ph, tt, off in parts:
            n = len(pos)
            s["h_pos"][off:off + n] = self.torch.from_numpy(np.ascontiguousarray(pos))
            s["h_ph"][off:off + n] = self.torch.from_numpy(np.ascontiguousarray(ph))
            s["h_t"][off:off + n] = self.torch.from_numpy(np.ascontiguousarray(tt))
        s["h_n"][0] = used
        s["count"] = used

    def launch(self, slot, used, chunks):
        """Replay the slot's graph, then copy each chunk's results straight into
        its own pinned host buffers (torch's caching host allocator), so results
        outlive the slot without any host-side copy."""
        torch = self.torch
        s = self.slots[slot]
        with torch.cuda.stream(s["stream"]):
            if s["graph"] is not None:
                s["graph"].replay()
            else:
                self._body(s)
            parts = []
            for off, count in chunks:
                part = {}
                for k in RESULT_KEYS:
                    src = s["out"][k][off:off + count]
                    part[k] = torch.empty(src.shape, dtype=src.dtype, pin_memory=True)
                    part[k].copy_(src, non_blocking=True)
                parts.append(part)
            s["status_host"] = torch.empty(4, dtype=torch.int32, pin_memory=True)
            s["status_host"].copy_(s["out"]["status"], non_blocking=True)
            s["parts"] = parts
            s["event"].record(s["stream"])

    def ready(self, slot):
        return self.slots[slot]["event"].query()

    def collect(self, slot):
        s = self.slots[slot]
        s["event"].synchronize()
        if int(s["status_host"][0]) & _lib.LH_STATUS_TIMEOUT:
            raise RuntimeError("a tensor-core pipeline wait timed out on the device")
        parts, s["parts"] = s["parts"], None
        return [{k: t.numpy() for k, t in part.items()} for part in parts]


def autotune(transport, n_flash, *, cache=None, candidates=(256, 512), repeats=5):
    """Pick the fused kernel's CTA size by timing each candidate once per shape.

    Results are cached in ``cache`` (a JSON file; default
    ``$LIGHTHIT_B200_AUTOTUNE`` or ``~/.cache/lighthit_b200/autotune.json``)
    under a key of device name, OM count, frequency and bin counts and mode.
    """
    import torch
    path = Path(cache or os.environ.get("LIGHTHIT_B200_AUTOTUNE",
                                        Path.home() / ".cache" / "lighthit_b200" / "autotune.json"))
    key = (f"{torch.cuda.get_device_name(transport.device)}|om{transport.n_om}|"
           f"w{transport.n_omega}|b{transport.n_bins}|{transport.mode}|n{n_flash}")
    table = {}
    if path.exists():
        try:
            table = json.loads(path.read_text())
        except (OSError, ValueError):
            table = {}
    if key in table:
        return int(table[key])
    n = max(1, int(n_flash))
    rng = np.random.default_rng(0)
    centre = transport.detector.positions_m.mean(axis=0)
    pos = torch.tensor(centre + rng.uniform(-40, 40, (n, 3)), dtype=torch.float64,
                       device=transport.device)
    ph = torch.full((n,), 1e10, dtype=torch.float64, device=transport.device)
    tt = torch.zeros(n, dtype=torch.float64, device=transport.device)
    out = transport.allocate(n)
    best, best_ms = candidates[-1], float("inf")
    for threads in candidates:
        transport.launch(pos, ph, tt, out, block_threads=threads)
        torch.cuda.synchronize(transport.device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            transport.launch(pos, ph, tt, out, block_threads=threads)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / repeats
        if ms < best_ms:
            best, best_ms = threads, ms
    table[key] = int(best)
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(".tmp")
        tmp.write_text(json.dumps(table, indent=1))
        os.replace(tmp, path)
    except OSError:
        pass
    return int(best)
