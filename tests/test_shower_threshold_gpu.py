"""Elements near the Cherenkov threshold on the device shower route (``-m gpu``).

Fixture: ``tests/golden/shower_threshold_c0.npz``
(``make_shower_threshold_golden.py``): the README shower with two fifths of its
elements slowed to emit in only one or two of the three wavelength nodes,
through the reference's float64 ``ShowerTransport``. Order 1 runs as a fused
unit plus one unit per band (``prompt.py:683-719``), the order >=2 source of
each node band compiles its own emitting elements (``shower/ge2.py:21-67``).
Tolerances as for the README shower.
"""
import numpy as np
import pytest

from conftest import GOLDEN

ORDER0, ORDER1, ORDER2 = 1e-4, 1e-5, 1e-4
BINS_L1 = 1e-3
FIELDS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
          "start_ns", "end_ns")
C_M_PER_NS = 0.299792458

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def routed():
    from lighthit_b200.shower import ShowerTables, ShowerTransport
    g = np.load(GOLDEN / "shower_threshold_c0.npz")
    el = np.load(GOLDEN / "order0_c0.npz")
    source = {k: np.asarray(el[k], float) for k in FIELDS}
    index = np.arange(len(source["beta"]))
    beta = source["beta"].copy()
    beta[index % 5 == 0] = float(g["beta_blue"])
    beta[index % 5 == 1] = float(g["beta_two"])
    source["beta"] = beta
    source["coefficient2"] = -source["coefficient0"] / beta ** 2
    source["end_ns"] = source["start_ns"] + source["length_m"] / (beta * C_M_PER_NS)
    tables = ShowerTables.synthetic("c0")
    return ShowerTransport(tables)(source), g, tables.threshold


def test_clocks_levels_and_active(routed):
    r, g, threshold = routed
    assert np.array_equal(r.time_origin_ns, g["time_origin_ns"])
    total = g["charge_components_pe"].sum(axis=1)
    near = np.abs(total - threshold) <= ORDER2 * np.maximum(np.abs(total), threshold)
    assert np.array_equal(r.active[~near], g["active"][~near])
    assert np.array_equal(np.asarray(r.metadata["ge2_charge_level"]), g["ge2_charge_level"])
    assert np.array_equal(np.asarray(r.metadata["prompt_order1_level"]), g["prompt_order1_level"])
    assert r.metadata["ge2_predictor"]["points"] == 15  # the reference's collapsed band-0 points
    assert not r.metadata["ge2_predictor"]["fallback_to_exact"]


def test_charge_per_order(routed):
    r, g, threshold = routed
    ref = g["charge_components_pe"]
    got = r.charge_components_pe
    total = ref.sum(axis=1)
    big = total >= threshold
    assert big.any()
    for order, tol in enumerate((ORDER0, ORDER1, ORDER2)):
        scale = np.abs(ref[big, order]) if order < 2 else np.abs(total[big])
        err = np.abs(got[big, order] - ref[big, order]) / np.maximum(scale, 1e-300)
        if order < 2:
            err = err[ref[big, order] > 1e-3 * total[big]]
        assert err.max(initial=0.0) <= tol, (order, err.max(initial=0.0))


def test_bins_and_spectrum(routed):
    r, g, _ = routed
    both = np.flatnonzero(r.active & g["active"])
    assert len(both)
    ref = g["components_pe"][both].astype(float)
    got = r.components_pe[both]
    charge = np.maximum(np.abs(g["charge_components_pe"][both]).sum(axis=1), 1e-300)
    for order in range(3):
        l1 = np.abs(got[:, :, order] - ref[:, :, order]).sum(axis=1) / charge
        assert l1.max() <= BINS_L1, (order, l1.max())
    spec_ref = g["spectrum_ge2_pe"][:, both]
    scale = np.abs(spec_ref).max(axis=0)
    assert (np.abs(r.spectrum_ge2_pe[:, both] - spec_ref).max(axis=0) / scale).max() < 1e-3
