"""Order 0 (direct light to the first glass entry): oracle pinned to the reference.

Fixtures: ``tests/golden/order0_c0.npz`` (``make_order0_golden.py``) and the
route's own order-0 charge and bins in ``shower_c0.npz`` (README-example
shower, 48 OMs, 2000 elements).
"""
import numpy as np
import pytest

from conftest import GOLDEN
from oracle import order0

ELEMENT_KEYS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
                "start_ns", "end_ns")
OPTICS_KEYS = ("panel_edges", "phase_nodes", "group_nodes", "extinction_nodes",
               "efficiency_coefficients")


def load():
    g = np.load(GOLDEN / "order0_c0.npz")
    det = dict(positions_m=g["positions_m"], looks=g["looks"], areas_m2=g["areas_m2"],
               radii_m=g["radii_m"], alpha=g["alpha"])
    el = {k: g[k] for k in ELEMENT_KEYS}
    optics = {k: g[k] for k in OPTICS_KEYS}
    return g, det, el, optics


def test_oracle_candidates_match_reference():
    g, det, el, optics = load()
    po, pe = order0.candidates(g["positions_m"], g["radii_m"], el["start_m"], el["direction"],
                               el["length_m"], el["coefficient0"], el["beta"], g["phase_nodes"])
    np.testing.assert_array_equal(po, g["pair_om"])
    np.testing.assert_array_equal(pe, g["pair_element"])


def test_oracle_rays_match_reference_at_order_8():
    g, det, el, optics = load()
    q, b = order0.rays(g["pair_om"], g["pair_element"], det, el, optics, g["origins_ns"],
                       g["edges_ns"], 8)
    assert np.abs(q - g["rays8_charge"]).max() <= 1e-12 * np.abs(g["rays8_charge"]).max()
    assert np.abs(b - g["rays8_bins"]).max() <= 1e-11 * np.abs(g["rays8_bins"]).max()
    sub = g["sub_pairs"]
    qs, bs = order0.rays(g["pair_om"][sub], g["pair_element"][sub], det, el, optics,
                         g["origins_ns"], g["edges_ns"], 8)
    assert np.abs(qs - g["sub8_charge"]).max() <= 1e-12 * np.abs(g["sub8_charge"]).max()
    assert np.abs(bs - g["sub8_bins"]).max() <= 1e-11 * np.abs(g["sub8_bins"]).max()


def test_ray_quadrature_converges_to_the_route():
    """Order-8 ray quadrature against the route's control-variate order 0.

    The route (``_surface_ballistic.py:114-353``) reaches its tolerance
    ``1e-10 + 2e-6 |q|`` by another rule; both approximate the same integral.
    """
    g, det, el, optics = load()
    s = np.load(GOLDEN / "shower_c0.npz")
    ref = s["charge_components_pe"][:, 0]
    q, b = order0.rays(g["pair_om"], g["pair_element"], det, el, optics, g["origins_ns"],
                       g["edges_ns"], 8)
    big = ref > 1e-3
    assert (np.abs(q - ref) / ref)[big].max() < 1e-7
    act = s["active"] & (ref > 0)
    l1 = np.abs(b[act] - s["components_pe"][act, :, 0]).sum(axis=1) / ref[act]
    assert l1.max() < 2e-4


def test_charge_only_edges_give_the_same_charge():
    """The route's charge-only call passes edges (-1e100, 1e100) and zero origins."""
    g, det, el, optics = load()
    sub = g["sub_pairs"]
    q, b = order0.rays(g["pair_om"][sub], g["pair_element"][sub], det, el, optics,
                       np.zeros(len(det["positions_m"])), np.array([-1e100, 1e100]), 8)
    assert np.abs(q - g["sub8_charge"]).max() <= 1e-7 * np.abs(g["sub8_charge"]).max()
    np.testing.assert_allclose(b[:, 0], q, rtol=1e-12, atol=0)


def test_oracle_rejects_a_segment_through_the_glass():
    g, det, el, optics = load()
    el2 = {k: np.array(v, copy=True) for k, v in el.items()}
    i = int(g["pair_element"][0])
    om = int(g["pair_om"][0])
    el2["start_m"][i] = g["positions_m"][om] - el2["direction"][i] * 0.05
    with pytest.raises(ValueError, match="intersects the glass"):
        order0.rays(np.array([om]), np.array([i]), det, el2, optics, g["origins_ns"],
                    g["edges_ns"], 8)
