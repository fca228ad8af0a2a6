"""Receiver subsets on the device shower route (``-m gpu``).

``ShowerTransport(tables)(source, receivers=ids)`` runs the route on those OMs
with threshold zero (``shower/api.py:205-212``): every receiver computed in
full, the response covering only them. Fixture:
``tests/golden/shower_receivers_c0.npz`` (``make_shower_receivers_golden.py``),
the README shower on seven OMs through the reference, with an event clock and
extra charges (``event``) and with the subset's own clock (``plain``).
Tolerances as for the README shower.
"""
import numpy as np
import pytest

from conftest import GOLDEN

ORDER0, ORDER1, ORDER2 = 1e-4, 1e-5, 1e-4
BINS_L1 = 1e-3
FIELDS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
          "start_ns", "end_ns")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def routed():
    from lighthit_b200.shower import ShowerTables, ShowerTransport
    g = np.load(GOLDEN / "shower_receivers_c0.npz")
    el = np.load(GOLDEN / "order0_c0.npz")
    source = {k: np.asarray(el[k], float) for k in FIELDS}
    route = ShowerTransport(ShowerTables.synthetic("c0"))
    ids = g["receivers"]
    out = {"event": route(source, receivers=ids, time_origin_ns=g["clock"],
                          selection_extra_charge=g["extra"]),
           "plain": route(source, receivers=ids)}
    return out, g, route


@pytest.mark.parametrize("name", ["event", "plain"])
def test_subset_response(routed, name):
    out, g, _ = routed
    r = out[name]
    n = len(g["receivers"])
    assert r.charge_components_pe.shape == (n, 3)
    assert np.array_equal(r.time_origin_ns, g[f"{name}_origin"])
    assert np.array_equal(r.active, g[f"{name}_active"])
    assert np.array_equal(np.asarray(r.metadata["ge2_charge_level"]), g[f"{name}_level"])
    ref = g[f"{name}_charge"]
    total = np.abs(ref).sum(axis=1)
    for order, tol in enumerate((ORDER0, ORDER1, ORDER2)):
        err = np.abs(r.charge_components_pe[:, order] - ref[:, order]) / total
        assert err.max() <= tol, (name, order, err.max())
    both = np.flatnonzero(r.active)
    for order in range(3):
        l1 = (np.abs(r.components_pe[both, :, order] - g[f"{name}_components"][both, :, order])
              .sum(axis=1) / total[both])
        assert l1.max() <= BINS_L1, (name, order, l1.max())
    spec_ref = g[f"{name}_spectrum"]
    scale = np.abs(spec_ref).max(axis=0)
    assert (np.abs(r.spectrum_ge2_pe - spec_ref).max(axis=0) / scale).max() < 1e-3


def test_subset_equals_full_route_on_active_oms(routed):
    """With the full response's clock, OMs active in the full route (computed in
    full there too) carry the same charges and bins in the subset."""
    _, g, route = routed
    el = np.load(GOLDEN / "order0_c0.npz")
    source = {k: np.asarray(el[k], float) for k in FIELDS}
    full = route(source)
    ids = g["receivers"]
    sub = route(source, receivers=ids, time_origin_ns=full.time_origin_ns[ids])
    keep = full.active[ids]
    assert keep.any()
    assert np.allclose(sub.charge_components_pe[keep], full.charge_components_pe[ids][keep],
                       rtol=1e-9, atol=1e-12)
    assert np.allclose(sub.components_pe[keep], full.components_pe[ids][keep],
                       rtol=1e-6, atol=1e-9)
