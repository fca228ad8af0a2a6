"""Serving loop: admission, splitting, ordering (host fake) and the device path."""
import numpy as np
import pytest

from lighthit_b200.serve import RESULT_KEYS, FlashServer, ServeConfig, flash_bytes


class FakeBackend:
    """Host stand-in: the 'kernel' writes values derived from each flash's inputs,
    and a launch completes after ``delay`` polls."""

    def __init__(self, capacity=5, n_slots=2, delay=2, n_om=3):
        self.capacity, self.n_slots, self.delay, self.n_om = capacity, n_slots, delay, n_om
        self.staged = {}
        self.clock = {}
        self.launch_sizes = []

    def stage(self, slot, parts, used):
        buf = np.zeros((used, 5))
        for pos, ph, tt, off in parts:
            buf[off:off + len(pos), :3] = pos
            buf[off:off + len(pos), 3] = ph
            buf[off:off + len(pos), 4] = tt
        self.staged[slot] = buf

    def launch(self, slot, used, chunks):
        self.launch_sizes.append(used)
        self.clock[slot] = self.delay
        self.chunks = getattr(self, "chunks", {})
        self.chunks[slot] = chunks

    def ready(self, slot):
        self.clock[slot] -= 1
        return self.clock[slot] <= 0

    def collect(self, slot):
        buf = self.staged[slot]
        n = len(buf)
        charge = buf[:, 3:4, None] * np.arange(1, self.n_om + 1)[None, :, None] * np.ones(3)
        active = np.ones((n, self.n_om), np.uint8)
        active[buf[:, 3] < 0] |= 2  # a negative photon count plays an unsafe flash
        out = dict(spectrum=np.repeat(buf[:, None, :3], self.n_om, 1), components=buf[:, None, :],
                   charge=charge, origin=buf[:, 4:5] + np.zeros(self.n_om), active=active)
        return [{k: v[off:off + count] for k, v in out.items()} for off, count in self.chunks[slot]]


def test_requests_split_batched_and_reassembled_in_order():
    be = FakeBackend(capacity=5, n_slots=2)
    srv = FlashServer(backend=be)
    rng = np.random.default_rng(0)
    reqs = []
    for n in (3, 7, 1, 5, 2, 11):
        pos = rng.normal(size=(n, 3))
        reqs.append((srv.submit(pos, rng.uniform(1, 2, n), rng.uniform(0, 5, n)), pos))
    srv.drain()
    assert max(be.launch_sizes) <= 5 and sum(be.launch_sizes) == 29
    for req, pos in reqs:
        assert req.done is not None and req.error is None
        assert req.result["spectrum"].shape[0] == len(pos)
        np.testing.assert_array_equal(req.result["spectrum"][:, 0, :], pos)
        np.testing.assert_array_equal(req.result["charge"][:, 0, 0], req.photons)
        np.testing.assert_array_equal(req.result["origin"][:, 0], req.time_ns)
        assert req.result["active"].dtype == bool


def test_requests_arriving_during_a_launch_join_the_next_one():
    be = FakeBackend(capacity=8, n_slots=1, delay=3)
    srv = FlashServer(backend=be)
    a = srv.submit(np.zeros((4, 3)), 1.0)
    srv.poll()                       # a is on the "GPU"
    b = srv.submit(np.ones((3, 3)), 1.0)
    c = srv.submit(np.ones((2, 3)), 1.0)
    srv.poll()
    assert be.launch_sizes == [4]    # no free slot yet: b, c wait
    srv.drain()
    assert be.launch_sizes == [4, 5]  # b and c admitted together when the slot freed
    assert a.done <= b.done and b.done == c.done


def test_device_error_is_attributed_to_its_request():
    srv = FlashServer(backend=FakeBackend(capacity=4))
    good = srv.submit(np.zeros((2, 3)), 1.0)
    bad = srv.submit(np.zeros((3, 3)), [1.0, -1.0, 1.0])
    srv.drain()
    assert good.error is None
    assert bad.error is not None and "flash 1" in bad.error


def test_budget_sizes_slots():
    per = flash_bytes(48, 65, 160)
    assert per == 40 + 48 * (65 * 24 + 1920 + 24 + 8 + 1)
    assert set(RESULT_KEYS) == {"spectrum", "components", "charge", "origin", "active"}


@pytest.mark.gpu
def test_served_results_equal_alone_and_in_the_mix(flash_table, flash_config, tmp_path):
    """Each request's result is the same served in a mix of uneven requests as alone."""
    from lighthit_b200.flash import FlashTransport
    from lighthit_b200.model import synthetic_detector
    from lighthit_b200.workloads import flash_batch_sizes, flash_positions
    det = synthetic_detector()
    ft = FlashTransport(det, flash_config, flash_table, mode="split-bf16")
    srv = FlashServer(ft, ServeConfig(hbm_budget_bytes=2 * 300 * flash_bytes(48, 65, 160),
                                      slots=2, autotune_cache=str(tmp_path / "tune.json")))
    assert srv.capacity == 300
    pos = flash_positions(700, det.positions_m.mean(axis=0), seed=5, om_positions=det.positions_m)
    sizes = flash_batch_sizes(700, seed=6, low=1, high=120)
    bounds = np.concatenate([[0], np.cumsum(sizes)])
    reqs = []
    burst = len(sizes) // 2
    for i, (a, b) in enumerate(zip(bounds[:-1], bounds[1:])):
        reqs.append(srv.submit(pos[a:b], 1e10))
        if i >= burst:  # the first half arrives at once, the rest one by one
            srv.poll()
    srv.drain()
    assert srv.launches < len(reqs)  # the burst was coalesced into launches
    for req, (a, b) in zip(reqs, zip(bounds[:-1], bounds[1:])):
        alone = ft.run(pos[a:b], 1e10)
        for k in RESULT_KEYS:
            ref = alone[k].cpu().numpy()
            if k == "active":
                ref = (ref & 1).astype(bool)
            np.testing.assert_array_equal(req.result[k], ref, err_msg=k)
