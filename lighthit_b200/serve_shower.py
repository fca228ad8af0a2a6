"""Serving loop for showers: continuous batching over worker streams.

Each worker owns a ``ShowerTransport`` on its own device tables and
workspaces and its own CUDA stream. A free worker takes every queued request
(up to ``max_batch``) as one batch and runs the route stage by stage for the
whole batch (``ShowerTransport.batch``), so requests that arrive while others
are on the device join the next batch, the kernels of several batches overlap
on the device, and the host orchestrates one batch while the device runs
another. Admission is by HBM budget: a batch is cut where the estimated device
footprint of the requests in flight would exceed it. Every result equals the
shower run alone (the stages are per shower; only launches are shared).
"""
from __future__ import annotations

import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

__all__ = ["ShowerRequest", "ShowerServer", "shower_footprint_bytes"]


def shower_footprint_bytes(n_elements, n_om):
    """Device bytes one shower holds while in flight (tables excluded): element
    copies, ring-node tables of the pencil compression (23 moments per slot),
    pencil rows, and per-OM group tables of the grouped order 1."""
    nodes = 192 * max(int(n_elements), 1)
    slots = 1 << int(np.ceil(np.log2(max(nodes, 4096))))
    return int(12 * 8 * n_elements + slots * 24 * 8 + nodes * 20 * 8
               + n_om * 8192 * 27 * 8)


@dataclass
class ShowerRequest:
    source: object
    arrival: float = field(default_factory=time.perf_counter)
    result: object = None
    error: BaseException | None = None
    done_at: float = 0.0
    footprint: int = 0

    @property
    def latency(self):
        return self.done_at - self.arrival


class ShowerServer:
    """``workers`` threads, each with its own route, stream and workspaces."""

    def __init__(self, make_route, *, workers=4, max_batch=16, hbm_budget_bytes=32 << 30,
                 n_om=384):
        import torch
        self.n_om = n_om
        self.max_batch = int(max_batch)
        self.budget = int(hbm_budget_bytes)
        self.in_flight = 0
        self.lock = threading.Condition()
        self.queue = queue.Queue()
        self.completed = []
        self.routes = [make_route() for _ in range(workers)]
        self.streams = [torch.cuda.Stream() for _ in range(workers)]
        self.threads = [threading.Thread(target=self._work, args=(k,), daemon=True)
                        for k in range(workers)]
        self._stop = False
        for t in self.threads:
            t.start()

    def submit(self, source, *, arrival=None):
        req = ShowerRequest(source, arrival if arrival is not None else time.perf_counter())
        n = len(np.asarray(source["length_m"] if isinstance(source, dict) else
                           getattr(getattr(source, "elements", source), "length_m")))
        req.footprint = shower_footprint_bytes(n, self.n_om)
        self.queue.put(req)
        return req

    def _take(self):
        """Block for one request, then take what else is queued (up to ``max_batch``)."""
        first = self.queue.get()
        if first is None:
            return None
        batch = [first]
        while len(batch) < self.max_batch:
            try:
                nxt = self.queue.get_nowait()
            except queue.Empty:
                break
            if nxt is None:
                self.queue.put(None)
                break
            batch.append(nxt)
        return batch

    def _work(self, k):
        import torch
        route, stream = self.routes[k], self.streams[k]
        while True:
            batch = self._take()
            if batch is None:
                return
            footprint = sum(r.footprint for r in batch)
            with self.lock:  # admission by HBM budget
                while self.in_flight and self.in_flight + footprint > self.budget:
                    self.lock.wait()
                self.in_flight += footprint
            try:
                with torch.cuda.stream(stream):
                    results = route.batch([r.source for r in batch])
                    stream.synchronize()
                for r, res in zip(batch, results):
                    r.result = res
            except BaseException:  # noqa: BLE001 - rerun alone to attach the error to its request
                for r in batch:
                    try:
                        with torch.cuda.stream(stream):
                            r.result = route(r.source)
                            stream.synchronize()
                    except BaseException as exc:  # noqa: BLE001 - handed back to the client
                        r.error = exc
            done = time.perf_counter()
            with self.lock:
                self.in_flight -= footprint
                for r in batch:
                    r.done_at = done
                    self.completed.append(r)
                self.lock.notify_all()

    def drain(self, count):
        """Wait until ``count`` requests completed; return and clear them."""
        with self.lock:
            while len(self.completed) < count:
                self.lock.wait(timeout=60.0)
            done, self.completed = self.completed[:count], self.completed[count:]
        return done

    def close(self):
        for _ in self.threads:
            self.queue.put(None)
        for t in self.threads:
            t.join(timeout=30)
