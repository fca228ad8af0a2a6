"""The near-field oracle against the reference's outputs (CPU).

``oracle/near.py`` restates ``near_field_ge2`` (``near_field.py:91-171``); the
fixture ``tests/golden/shower_near_c0.npz`` holds the reference's own float64
results (``make_shower_near_golden.py``). The table is the first radial
interval of the per-wavelength splines (``lighthit_b200/tables/near_c0.npz``),
the rest of the constants the route's (``route_c0.npz``).
"""
import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from oracle.near import near_field

FIELDS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
          "start_ns", "end_ns")
TABLES = ROOT / "lighthit_b200" / "tables"


@pytest.fixture(scope="module")
def setup():
    table = dict(np.load(TABLES / "near_c0.npz"))
    route = np.load(TABLES / "route_c0.npz")
    kw = dict(wavelength_nm=route["wavelength_nm"], weight_nm=route["weight_nm"],
              efficiency=route["efficiency"], phase_index=route["phase_index"],
              alpha=route["alpha"])
    det = (route["positions_m"], route["looks"], route["areas_m2"])
    return table, det, kw, np.load(GOLDEN / "shower_near_c0.npz")


def _compare(result, oms, charge, spectrum, elements):
    got_oms, got_charge, got_spectrum, got_elements = result
    assert np.array_equal(got_oms, oms)
    assert got_elements == elements
    assert np.allclose(got_charge[oms], charge, rtol=1e-11, atol=0)
    scale = np.abs(spectrum).max(axis=0)
    assert (np.abs(got_spectrum[:, oms] - spectrum).max(axis=0) / scale).max() < 1e-11


def test_oracle_edge_cases(setup):
    table, det, kw, g = setup
    el = {k: g[f"edges_{k}"] for k in FIELDS}
    _compare(near_field(table, el, *det, g["edges_origins_ns"], **kw), g["edges_oms"],
             g["edges_charge_pe"], g["edges_spectrum_pe"], int(g["edges_elements"]))


def test_oracle_moved_shower(setup):
    table, det, kw, g = setup
    shower = np.load(GOLDEN / "order0_c0.npz")
    el = {k: np.asarray(shower[k], float) for k in FIELDS}
    el["start_m"] = el["start_m"] + g["shift_m"]
    _compare(near_field(table, el, *det, g["pass_time_origin_ns"], **kw), g["pass_near_oms"],
             g["pass_near_charge_pe"], g["pass_near_spectrum_pe"], int(g["pass_near_elements"]))
