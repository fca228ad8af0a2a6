"""Near-field clamp of order >=2 on the device against the reference (``-m gpu``).

Fixture: ``tests/golden/shower_near_c0.npz`` (``make_shower_near_golden.py``),
the reference's float64 ``near_field_ge2`` (``near_field.py:91-171``) and
``ShowerTransport`` with ``add_near_field`` (``near_field.py:174-217``):

* ``edges``: hand-made elements around two OMs (a line through an OM centre,
  portions clipped at either end, many panels, partial and absent cone
  harmonics) on a random per-OM clock, through ``lh_near_field`` alone;
* ``pass``: the README shower moved to pass 1 m from OM 20, the near field
  alone on the response clock and the whole route.

The kernel contracts in float32 (complex64 splines) and accumulates in
float64: spectra within 1e-5 of each OM's largest value, charges within 1e-5.
"""
import numpy as np
import pytest

from conftest import GOLDEN

FIELDS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
          "start_ns", "end_ns")
NEAR_TOL = 1e-5
ORDER0, ORDER1, ORDER2 = 1e-4, 1e-5, 1e-4
BINS_L1 = 1e-3

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN / "shower_near_c0.npz")


@pytest.fixture(scope="module")
def tables():
    from lighthit_b200.shower import ShowerTables
    return ShowerTables.synthetic("c0")


def _moved(g):
    el = np.load(GOLDEN / "order0_c0.npz")
    source = {k: np.asarray(el[k], float) for k in FIELDS}
    source["start_m"] = source["start_m"] + g["shift_m"]
    return source


def _near_alone(tables, source, origins):
    import torch
    dev = tables.device
    el = {k: torch.tensor(np.ascontiguousarray(source[k], float), dtype=torch.float64, device=dev)
          for k in FIELDS}
    o = torch.tensor(np.asarray(origins, float), dtype=torch.float64, device=dev)
    return tables.near.field(el, len(source["beta"]), tables._pos, tables._looks,
                             tables._areas, o)


def _check_near(near, oms, charge, spectrum, elements):
    assert np.array_equal(near.oms, oms)
    assert near.metadata["elements"] == elements
    got = near.charge_pe[oms]
    assert np.abs(got - charge).max() <= NEAR_TOL * np.abs(charge).max()
    spec = near.spectrum.cpu().numpy()[oms].T
    scale = np.abs(spectrum).max(axis=0)
    assert (np.abs(spec - spectrum).max(axis=0) / scale).max() <= NEAR_TOL


def test_near_field_edge_cases(golden, tables):
    g = golden
    source = {k: g[f"edges_{k}"] for k in FIELDS}
    near = _near_alone(tables, source, g["edges_origins_ns"])
    _check_near(near, g["edges_oms"], g["edges_charge_pe"], g["edges_spectrum_pe"],
                int(g["edges_elements"]))
    # OMs without portions get exact zeros
    rest = np.setdiff1d(np.arange(tables.n_om), g["edges_oms"])
    assert not np.any(near.charge_pe[rest])
    assert not np.any(near.spectrum.cpu().numpy()[rest])


def test_near_field_of_the_moved_shower(golden, tables):
    g = golden
    near = _near_alone(tables, _moved(g), g["pass_time_origin_ns"])
    _check_near(near, g["pass_near_oms"], g["pass_near_charge_pe"], g["pass_near_spectrum_pe"],
                int(g["pass_near_elements"]))


@pytest.fixture(scope="module")
def routed(golden, tables):
    from lighthit_b200.shower import ShowerTransport
    with pytest.warns(RuntimeWarning, match="near-field clamp"):
        return ShowerTransport(tables)(_moved(golden))


def test_route_near_record(golden, routed):
    g = golden
    (record,) = routed.metadata["near_field"]
    assert record["oms"] == g["pass_near_oms"].tolist()
    assert record["elements"] == int(g["pass_near_elements"])
    assert record["bins_added_oms"] == g["pass_near_bins_added"].tolist()
    ref = g["pass_near_charge_pe"]
    assert np.abs(np.array(record["charge_pe"]) - ref).max() <= NEAR_TOL * np.abs(ref).max()


def test_route_clocks_and_active(golden, tables, routed):
    g = golden
    assert np.array_equal(routed.time_origin_ns, g["pass_time_origin_ns"])
    total = g["pass_charge_components_pe"].sum(axis=1)
    near = np.abs(total - tables.threshold) <= ORDER2 * np.maximum(np.abs(total),
                                                                   tables.threshold)
    assert np.array_equal(routed.active[~near], g["pass_active"][~near])


def test_route_charge_per_order(golden, tables, routed):
    ref = golden["pass_charge_components_pe"]
    got = routed.charge_components_pe
    total = ref.sum(axis=1)
    big = total >= tables.threshold
    assert big.any()
    for order, tol in enumerate((ORDER0, ORDER1, ORDER2)):
        scale = np.abs(ref[big, order]) if order < 2 else np.abs(total[big])
        err = np.abs(got[big, order] - ref[big, order]) / np.maximum(scale, 1e-300)
        if order < 2:
            err = err[ref[big, order] > 1e-3 * total[big]]
        assert err.max(initial=0.0) <= tol, (order, err.max(initial=0.0))
    om = int(golden["om"])  # the near OM itself, every order
    err = np.abs(got[om] - ref[om]) / np.abs(ref[om]).sum()
    assert err.max() <= ORDER2, err


def test_route_bins_and_spectrum(golden, routed):
    g = golden
    both = np.flatnonzero(routed.active & g["pass_active"])
    assert int(g["om"]) in both
    ref = g["pass_components_pe"][both].astype(float)
    got = routed.components_pe[both]
    charge = np.maximum(np.abs(g["pass_charge_components_pe"][both]).sum(axis=1), 1e-300)
    for order in range(3):
        l1 = np.abs(got[:, :, order] - ref[:, :, order]).sum(axis=1) / charge
        assert l1.max() <= BINS_L1, (order, l1.max())
    spec_ref = g["pass_spectrum_ge2_pe"][:, both]
    scale = np.abs(spec_ref).max(axis=0)
    assert (np.abs(routed.spectrum_ge2_pe[:, both] - spec_ref).max(axis=0) / scale).max() < 1e-3
