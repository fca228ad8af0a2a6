"""Delayed light on the device shower route against the reference (``-m gpu``).

Fixture: ``tests/golden/shower_delayed_c0.npz`` (``make_shower_delayed_golden.py``):
the README shower plus delayed copies of some of its steps (delayed groups
inside the readout window, steps beyond it), through the reference's
float64 ``ShowerTransport``. The route splits the steps with ``delay_groups``
(``shower/ge2.py:122-147``): prompt steps make the stored spectrum, every
delayed step adds its exact zero-frequency >=2 charge, and each group inside
the window adds bins read on its own clock (``shower/api.py:438-477``).
Tolerances as for the prompt-only README shower.
"""
import numpy as np
import pytest

from conftest import GOLDEN

ORDER0 = 1e-4
ORDER1 = 1e-5
ORDER2 = 1e-4
BINS_L1 = 1e-3
FIELDS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
          "start_ns", "end_ns")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def delayed():
    from lighthit_b200.shower import ShowerTables, ShowerTransport
    g = np.load(GOLDEN / "shower_delayed_c0.npz")
    el = np.load(GOLDEN / "order0_c0.npz")
    base = {k: np.asarray(el[k]) for k in FIELDS}
    parts = [np.arange(len(base["beta"])), g["delayed_a"], g["beyond"]]
    delays = [0.0, *[float(d) for d in g["delays"]]]
    source = {k: np.concatenate([base[k][idx] + (d if k.endswith("_ns") else 0.0)
                                 for idx, d in zip(parts, delays)]) for k in FIELDS}
    route = ShowerTransport(ShowerTables.synthetic("c0"))
    return route(source), g, route.tables.threshold


def test_delay_groups_match(delayed):
    r, g, _ = delayed
    meta = r.metadata["delayed_light"]
    assert meta["groups_in_window"] == int(g["groups_in_window"])
    assert meta["steps_beyond_window"] == int(g["steps_beyond_window"])
    ref = float(g["delayed_charge_pe"])
    assert abs(meta["delayed_charge_pe"] - ref) <= ORDER2 * max(abs(ref), 1e-3)


def test_clocks_and_active(delayed):
    r, g, threshold = delayed
    assert np.array_equal(r.time_origin_ns, g["time_origin_ns"])
    total = g["charge_components_pe"].sum(axis=1)
    near = np.abs(total - threshold) <= ORDER2 * np.maximum(np.abs(total), threshold)
    assert np.array_equal(r.active[~near], g["active"][~near])


def test_charge_per_order(delayed):
    r, g, threshold = delayed
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


def test_bins_and_spectrum(delayed):
    r, g, _ = delayed
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
