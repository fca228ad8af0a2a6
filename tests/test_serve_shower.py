"""Shower serving loop on the host: admission by HBM budget, batching, errors,
bounded waits (a fake route stands in for the device route)."""
import threading
import time

import pytest

from lighthit_b200.serve_shower import ShowerServer


class FakeRoute:
    """``batch`` doubles each source's value after ``delay`` seconds and records
    the batches it saw; a source with ``bad`` raises."""

    def __init__(self, delay=0.01, gate=None):
        self.delay = delay
        self.gate = gate
        self.batches = []

    def batch(self, sources):
        if self.gate is not None:
            self.gate.wait()
        self.batches.append([s["id"] for s in sources])
        time.sleep(self.delay)
        if any(s.get("bad") for s in sources):
            raise ValueError("bad shower")
        return [2 * s["value"] for s in sources]

    def __call__(self, source):
        return self.batch([source])[0]


def server(routes, **kw):
    it = iter(routes)
    kw.setdefault("footprint", lambda s: s["bytes"])
    return ShowerServer(lambda: next(it), workers=len(routes), device_streams=False, **kw)


def test_results_in_order_and_batched():
    routes = [FakeRoute(), FakeRoute()]
    srv = server(routes, max_batch=4, hbm_budget_bytes=1000)
    reqs = [srv.submit({"id": k, "value": k, "bytes": 10}) for k in range(30)]
    done = srv.drain(30, timeout=30)
    srv.close()
    assert len(done) == 30
    for r in reqs:
        assert r.error is None and r.result == 2 * r.source["value"]
    sizes = [len(b) for rt in routes for b in rt.batches]
    assert max(sizes) <= 4 and sum(sizes) == 30


def test_admission_keeps_the_footprint_in_flight_under_the_budget():
    routes = [FakeRoute(delay=0.02) for _ in range(3)]
    srv = server(routes, max_batch=8, hbm_budget_bytes=100)
    for k in range(40):
        srv.submit({"id": k, "value": k, "bytes": 30})
    srv.drain(40, timeout=30)
    srv.close()
    assert srv.peak_in_flight <= 100
    assert max(len(b) for rt in routes for b in rt.batches) <= 3  # 3 x 30 bytes fit, 4 do not


def test_a_request_above_the_budget_runs_alone():
    routes = [FakeRoute(), FakeRoute()]
    srv = server(routes, max_batch=8, hbm_budget_bytes=100)
    srv.submit({"id": 0, "value": 1, "bytes": 500})
    for k in range(1, 6):
        srv.submit({"id": k, "value": k, "bytes": 10})
    done = srv.drain(6, timeout=30)
    srv.close()
    assert all(r.error is None for r in done)
    big = [b for rt in routes for b in rt.batches if 0 in b]
    assert big == [[0]]


def test_a_failing_request_gets_its_error_and_the_others_their_results():
    route = FakeRoute()
    srv = server([route], max_batch=8, hbm_budget_bytes=1000)
    gate_reqs = [srv.submit({"id": k, "value": k, "bytes": 1, "bad": k == 3}) for k in range(6)]
    srv.drain(6, timeout=30)
    srv.close()
    for r in gate_reqs:
        if r.source["id"] == 3:
            assert isinstance(r.error, ValueError) and r.result is None
        else:
            assert r.error is None and r.result == 2 * r.source["value"]


def test_drain_is_bounded():
    gate = threading.Event()
    srv = server([FakeRoute(gate=gate)], max_batch=2, hbm_budget_bytes=1000)
    srv.submit({"id": 0, "value": 0, "bytes": 1})
    with pytest.raises(TimeoutError):
        srv.drain(1, timeout=0.2)
    gate.set()
    assert len(srv.drain(1, timeout=30)) == 1
    srv.close()


def test_base_exceptions_are_handed_back_to_the_request():
    class Broken(FakeRoute):
        def batch(self, sources):
            raise SystemExit("worker gone")  # BaseException past the per-request rerun

        def __call__(self, source):
            raise SystemExit("worker gone")

    srv = server([Broken()], max_batch=2, hbm_budget_bytes=1000)
    srv.submit({"id": 0, "value": 0, "bytes": 1})
    # the per-request rerun attaches the error to the request; the worker lives on
    done = srv.drain(1, timeout=30)
    assert isinstance(done[0].error, SystemExit)
    srv.close()


def test_prime_runs_the_sources_on_every_worker_in_batches():
    routes = [FakeRoute(delay=0.0) for _ in range(3)]
    srv = server(routes, max_batch=4, hbm_budget_bytes=1000)
    srv.prime([{"id": k, "value": k, "bytes": 10} for k in range(6)])
    for rt in routes:
        assert rt.batches == [[0, 1, 2, 3], [4, 5]]
    assert srv.completed == []  # priming hands nothing to drain()
    reqs = [srv.submit({"id": k, "value": k, "bytes": 10}) for k in range(5)]
    srv.drain(5, timeout=30)
    srv.close()
    assert [r.result for r in reqs] == [2 * k for k in range(5)]


def test_prime_refuses_once_requests_are_queued():
    gate = threading.Event()
    srv = server([FakeRoute(gate=gate)], max_batch=2, hbm_budget_bytes=1000)
    srv.submit({"id": 0, "value": 0, "bytes": 10})
    with pytest.raises(RuntimeError):
        srv.prime([{"id": 1, "value": 1, "bytes": 10}])
    gate.set()
    srv.drain(1, timeout=30)
    srv.close()
