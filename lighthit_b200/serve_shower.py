"""Serving loop for showers: continuous batching over worker streams.

Each worker owns a ``ShowerTransport`` on its own device tables and
workspaces and its own CUDA stream. A free worker takes the queued requests
(up to ``max_batch``, cut where their estimated device footprint would pass
the HBM budget left) as one batch and runs the route stage by stage for the
whole batch (``ShowerTransport.batch``), so requests that arrive while others
are on the device join the next batch, the kernels of several batches overlap
on the device, and the host orchestrates one batch while the device runs
another. A batch waits for admission while the footprint of the batches in
flight plus its own would pass the budget; one request larger than the whole
budget runs alone. Every result equals the shower run alone (the stages are
per shower; only launches are shared).
"""
from __future__ import annotations

import threading
import time
from collections import deque
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


def _element_count(source):
    el = source if isinstance(source, dict) else getattr(source, "elements", source)
    return len(np.asarray(el["length_m"] if isinstance(el, dict) else getattr(el, "length_m")))


@dataclass
class ShowerRequest:
    source: object
    arrival: float = field(default_factory=time.perf_counter)
    result: object = None
    error: BaseException | None = None
    done_at: float = 0.0
    footprint: int = 0
    batch_size: int = 0

    @property
    def latency(self):
        return self.done_at - self.arrival


class ShowerServer:
    """``workers`` threads, each with its own route, stream and workspaces.

    ``make_route()`` returns an object with ``batch(sources)`` (and
    ``__call__(source)`` for the rerun of a failed batch one request at a
    time); ``footprint(source)`` overrides ``shower_footprint_bytes``.
    """

    def __init__(self, make_route, *, workers=4, max_batch=16, hbm_budget_bytes=32 << 30,
                 n_om=384, footprint=None, device_streams=True):
        self.n_om = n_om
        self.max_batch = int(max_batch)
        self.budget = int(hbm_budget_bytes)
        self.in_flight = 0
        self.peak_in_flight = 0
        self.lock = threading.Condition()
        self.pending = deque()
        self.completed = []
        self._footprint = footprint or (lambda s: shower_footprint_bytes(_element_count(s), n_om))
        self.routes = [make_route() for _ in range(workers)]
        if device_streams:
            import torch
            self.streams = [torch.cuda.Stream() for _ in range(workers)]
        else:
            self.streams = [None] * workers
        self._stop = False
        self.worker_errors = []
        self.threads = [threading.Thread(target=self._work, args=(k,), daemon=True)
                        for k in range(workers)]
        for t in self.threads:
            t.start()

    def prime(self, sources):
        """Run ``sources`` once on every worker, before serving (results dropped).

        A worker's route grows its device workspaces and tables (pencil and
        group tables, source lattices) to the largest shower it has seen, and
        the allocator keeps freed blocks per stream; a shower larger than any
        before it therefore allocates device memory in the middle of serving.
        Priming with the largest showers expected (as many copies as the route
        has side-stream lanes, so that every lane sees them) sizes all of that
        up front."""
        sources = list(sources)
        if not sources:
            return
        with self.lock:
            if self.in_flight or self.pending:
                raise RuntimeError("prime() runs before any request is submitted")
        for route, stream in zip(self.routes, self.streams):
            for first in range(0, len(sources), self.max_batch):
                self._run(route, stream, sources[first:first + self.max_batch])

    def submit(self, source, *, arrival=None):
        req = ShowerRequest(source, arrival if arrival is not None else time.perf_counter())
        req.footprint = int(self._footprint(source))
        with self.lock:
            if self._stop:
                raise RuntimeError("the server is closed")
            self.pending.append(req)
            self.lock.notify_all()
        return req

    def _take(self):
        """Wait for work and admission; return the next batch (None on close).

        The batch takes queued requests in arrival order up to ``max_batch``
        while their footprint fits the budget left by the batches in flight;
        with nothing in flight the first request is always admitted."""
        with self.lock:
            while True:
                if self._stop and not self.pending:
                    return None
                if self.pending:
                    room = self.budget - self.in_flight
                    batch, total = [], 0
                    while self.pending and len(batch) < self.max_batch:
                        f = self.pending[0].footprint
                        if total + f > room and (batch or self.in_flight):
                            break
                        batch.append(self.pending.popleft())
                        total += f
                    if batch:
                        self.in_flight += total
                        self.peak_in_flight = max(self.peak_in_flight, self.in_flight)
                        return batch, total
                self.lock.wait()

    def _run(self, route, stream, sources):
        if stream is None:
            return route.batch(sources)
        import torch
        with torch.cuda.stream(stream):
            out = route.batch(sources)
            stream.synchronize()
        return out

    def _run_one(self, route, stream, source):
        if stream is None:
            return route(source)
        import torch
        with torch.cuda.stream(stream):
            out = route(source)
            stream.synchronize()
        return out

    def _work(self, k):
        route, stream = self.routes[k], self.streams[k]
        try:
            while True:
                taken = self._take()
                if taken is None:
                    return
                batch, footprint = taken
                try:
                    results = self._run(route, stream, [r.source for r in batch])
                    for r, res in zip(batch, results):
                        r.result = res
                except BaseException:  # noqa: BLE001 - rerun alone to attach the error to its request
                    for r in batch:
                        try:
                            r.result = self._run_one(route, stream, r.source)
                        except BaseException as exc:  # noqa: BLE001 - handed back to the client
                            r.error = exc
                done = time.perf_counter()
                with self.lock:
                    self.in_flight -= footprint
                    for r in batch:
                        r.done_at = done
                        r.batch_size = len(batch)
                        self.completed.append(r)
                    self.lock.notify_all()
        except BaseException as exc:  # noqa: BLE001 - a dead worker is reported by drain()
            with self.lock:
                self.worker_errors.append(exc)
                self.lock.notify_all()

    def drain(self, count, *, timeout=600.0):
        """Wait until ``count`` requests completed; return and clear them.

        Raises ``TimeoutError`` when they have not completed within ``timeout``
        seconds, and ``RuntimeError`` when a worker thread died."""
        deadline = time.perf_counter() + float(timeout)
        with self.lock:
            while len(self.completed) < count:
                if self.worker_errors:
                    raise RuntimeError("a shower worker died") from self.worker_errors[0]
                if not any(t.is_alive() for t in self.threads):
                    raise RuntimeError("no shower worker is running")
                left = deadline - time.perf_counter()
                if left <= 0:
                    raise TimeoutError(f"{len(self.completed)} of {count} showers completed "
                                       f"within {timeout:g} s")
                self.lock.wait(timeout=min(left, 1.0))
            done, self.completed = self.completed[:count], self.completed[count:]
        return done

    def close(self, timeout=30.0):
        with self.lock:
            self._stop = True
            self.lock.notify_all()
        for t in self.threads:
            t.join(timeout=timeout)
