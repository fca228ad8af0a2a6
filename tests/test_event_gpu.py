"""A two-shower event on the device routes against the reference (``-m gpu``).

Fixture: ``tests/golden/event_c0.npz`` (``make_event_golden.py``): the
reference ``EventTransport`` (``event.py:94-296``) on the README shower and a
moved, delayed copy of it: one clock for the event, each source's threshold
decisions with the other's charge, completion rounds on receiver subsets.
Tolerances as for the README shower; the completion rounds recompute the same
OMs.
"""
import json

import numpy as np
import pytest

from conftest import GOLDEN

ORDER0, ORDER1, ORDER2 = 1e-4, 1e-5, 1e-4
BINS_L1 = 1e-3
FIELDS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
          "start_ns", "end_ns")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def event():
    from lighthit_b200.event import EventTransport, SourceComponent
    from lighthit_b200.shower import ShowerTables, ShowerTransport
    g = np.load(GOLDEN / "event_c0.npz")
    el = np.load(GOLDEN / "order0_c0.npz")
    first = {k: np.asarray(el[k], float) for k in FIELDS}
    second = dict(first, start_m=first["start_m"] + g["shift_m"],
                  start_ns=first["start_ns"] + float(g["delay_ns"]),
                  end_ns=first["end_ns"] + float(g["delay_ns"]))
    route = ShowerTransport(ShowerTables.synthetic("c0"))
    r = EventTransport(route)([SourceComponent("shower", first, label="a"),
                               SourceComponent("shower", second, label="b")])
    return r, g, route.tables.threshold


def test_event_clock_mask_and_rounds(event):
    r, g, threshold = event
    assert np.array_equal(r.time_origin_ns, g["time_origin_ns"])
    total = g["charge_components_pe"].sum(axis=1)
    near = np.abs(total - threshold) <= ORDER2 * np.maximum(np.abs(total), threshold)
    assert np.array_equal(r.active[~near], g["active"][~near])
    ref_rounds = json.loads(str(g["rounds"]))
    got = [dict(x["recomputed"]) for x in r.metadata["completion_rounds"]]
    assert got == [dict(x["recomputed"]) for x in ref_rounds]


def test_event_charge_bins_and_spectrum(event):
    r, g, threshold = event
    ref = g["charge_components_pe"]
    total = ref.sum(axis=1)
    big = total >= threshold
    for order, tol in enumerate((ORDER0, ORDER1, ORDER2)):
        scale = np.abs(ref[big, order]) if order < 2 else np.abs(total[big])
        err = np.abs(r.charge_components_pe[big, order] - ref[big, order]) / np.maximum(scale, 1e-300)
        if order < 2:
            err = err[ref[big, order] > 1e-3 * total[big]]
        assert err.max(initial=0.0) <= tol, (order, err.max(initial=0.0))
    both = np.flatnonzero(r.active & g["active"])
    charge = np.abs(ref[both]).sum(axis=1)
    for order in range(3):
        l1 = np.abs(r.components_pe[both, :, order]
                    - g["components_pe"][both, :, order]).sum(axis=1) / charge
        assert l1.max() <= BINS_L1, (order, l1.max())
    spec_ref = g["spectrum_ge2_pe"][:, both]
    scale = np.abs(spec_ref).max(axis=0)
    assert (np.abs(r.spectrum_ge2_pe[:, both] - spec_ref).max(axis=0) / scale).max() < 1e-3
