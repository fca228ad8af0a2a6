"""Config 2 (384 OMs, 2-450 m tables): the device route against the reference's
own float64 ``ShowerTransport`` on the first 12 showers of the seeded stream
(``-m gpu``).

Fixture: ``tests/golden/shower_c2.npz`` (``make_shower_c2_golden.py``). The 12
showers run as one stage-major batch (the serving path). Tolerances as for the
README shower: per-order charge relative to the reference's per-OM charge for
OMs at or above threshold (order 0 ORDER0, order 1 ORDER1, order >=2 ORDER2 of
the OM's total), per-order bin L1 BINS_L1 of the OM's charge, clocks
bit-identical, the active mask identical away from threshold (an OM within
ORDER2 of ``threshold_pe`` may flip).
"""
import numpy as np
import pytest

from conftest import GOLDEN

ORDER0 = 1e-4
ORDER1 = 1e-5
ORDER2 = 1e-4
BINS_L1 = 1e-3
N_SHOWERS = 12

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def routed():
    from lighthit_b200.shower import ShowerTables, ShowerTransport
    from lighthit_b200.workloads import gaussian_shower, shower_stream
    g = np.load(GOLDEN / "shower_c2.npz")
    route = ShowerTransport(ShowerTables.synthetic("c2"))
    stream = shower_stream(N_SHOWERS, route.tables.positions.mean(axis=0))
    sources = []
    for k, s in enumerate(stream):
        el = gaussian_shower(s["position_m"], s["direction"],
                             charged_track_length_m=s["charged_track_length_m"],
                             elements=s["elements"], seed=s["seed"])
        assert int(g[f"s{k}_elements"]) == s["elements"]
        assert float(el["start_m"].sum() + el["start_ns"].sum()) == float(g[f"s{k}_checksum"])
        sources.append(el)
    return route.batch(sources), g, route.tables.threshold


def test_clocks_bit_identical(routed):
    responses, g, _ = routed
    for k, r in enumerate(responses):
        assert np.array_equal(r.time_origin_ns, g[f"s{k}_origin"]), k


def test_active_mask(routed):
    responses, g, threshold = routed
    for k, r in enumerate(responses):
        ref = g[f"s{k}_active"]
        total = g[f"s{k}_charge"].sum(axis=1)
        near = np.abs(total - threshold) <= ORDER2 * np.maximum(np.abs(total), threshold)
        assert np.array_equal(r.active[~near], ref[~near]), k


def test_charge_per_order(routed):
    responses, g, threshold = routed
    worst = np.zeros(3)
    for k, r in enumerate(responses):
        ref = g[f"s{k}_charge"]
        got = r.charge_components_pe
        total = ref.sum(axis=1)
        big = total >= threshold
        if not big.any():
            continue
        for order, tol in enumerate((ORDER0, ORDER1, ORDER2)):
            scale = np.abs(ref[big, order]) if order < 2 else np.abs(total[big])
            err = np.abs(got[big, order] - ref[big, order]) / np.maximum(scale, 1e-300)
            if order < 2:
                err = err[ref[big, order] > 1e-3 * total[big]]
            worst[order] = max(worst[order], err.max(initial=0.0))
            assert err.max(initial=0.0) <= tol, (k, order, err.max())
    print("worst per-order relative charge error", worst)


def test_bins_per_order(routed):
    responses, g, _ = routed
    for k, r in enumerate(responses):
        ids = g[f"s{k}_active_ids"]
        if not len(ids):
            continue
        both = ids[r.active[ids]]
        pos = np.searchsorted(ids, both)
        ref = g[f"s{k}_components"][pos].astype(float)
        got = r.components_pe[both]
        charge = np.maximum(np.abs(g[f"s{k}_charge"][both]).sum(axis=1), 1e-300)
        for order in range(3):
            l1 = np.abs(got[:, :, order] - ref[:, :, order]).sum(axis=1) / charge
            assert l1.max() <= BINS_L1, (k, order, l1.max())


def test_coarse_only_order1_charge(routed):
    """OMs the coarse screen left below threshold keep the screen's charge
    (compress_screen / screen_order1: parents refined near the OM, the two-node
    radial rule): equal to the reference's coarse charge."""
    responses, g, _ = routed
    seen = 0
    for k, r in enumerate(responses):
        level = np.asarray(r.metadata["prompt_order1_level"])
        coarse = level == 1
        ref = g[f"s{k}_charge"][coarse, 1]
        got = r.charge_components_pe[coarse, 1]
        scale = np.maximum(np.abs(ref), 1e-12)
        assert (np.abs(got - ref) / scale).max(initial=0.0) <= ORDER1, k
        seen += int(coarse.sum())
    assert seen > 100
