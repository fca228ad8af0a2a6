"""The served shower loop on the device: every result equals the shower routed
alone, with requests arriving while other batches run on the device."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_served_showers_equal_each_shower_alone():
    from lighthit_b200.serve_shower import ShowerServer
    from lighthit_b200.shower import ShowerTables, ShowerTransport
    from lighthit_b200.workloads import gaussian_shower, shower_stream
    alone_route = ShowerTransport(ShowerTables.synthetic("c2"))
    draws = shower_stream(10, alone_route.tables.positions.mean(axis=0))
    showers = [gaussian_shower(d["position_m"], d["direction"],
                               charged_track_length_m=d["charged_track_length_m"],
                               elements=min(d["elements"], 6000), seed=d["seed"]) for d in draws]
    server = ShowerServer(lambda: ShowerTransport(ShowerTables.synthetic("c2")), workers=2,
                          max_batch=3)
    try:
        # workspaces sized by the largest showers first: results are unchanged
        server.prime(sorted(showers, key=lambda s: len(s["length_m"]))[-2:] * 2)
        assert server.completed == []
        early = [server.submit(s) for s in showers[:4]]
        time.sleep(0.05)  # the first batches are on the device when the rest arrive
        late = [server.submit(s) for s in showers[4:]]
        done = server.drain(len(showers), timeout=600)
    finally:
        server.close()
    assert len(done) == len(showers)
    assert max(r.batch_size for r in done) > 1  # some showers were served in a mix
    for req, src in zip(early + late, showers):
        assert req.error is None, req.error
        got, alone = req.result, alone_route(src)
        assert np.array_equal(got.active, alone.active)
        assert np.array_equal(got.time_origin_ns, alone.time_origin_ns)
        # orders 0 and 1 add per-block float64 partial sums with atomics, whose
        # order depends on what else shares the launch: a few 1e-16 per term
        scale = max(np.abs(alone.charge_pe).max(), 1e-300)
        assert np.abs(got.charge_components_pe - alone.charge_components_pe).max() <= 1e-10 * scale
        assert np.abs(got.components_pe - alone.components_pe).max() <= 1e-10 * scale
        assert got.metadata["ge2_charge_level"] == alone.metadata["ge2_charge_level"]
