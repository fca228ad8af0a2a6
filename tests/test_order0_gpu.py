"""Order 0 on the device against the oracle and the reference (``-m gpu``).

Tolerances: the device evaluates the same ray quadrature as the oracle at the
same Gauss order, with the innermost azimuth integrand in float32; per-OM
charge agrees to ORDER0_CHARGE_TOL relative and the bins to ORDER0_BINS_TOL
of the OM's charge (L1).
"""
import numpy as np
import pytest

from conftest import GOLDEN
from oracle import order0 as oracle

ORDER0_CHARGE_TOL = 2e-5
ORDER0_BINS_TOL = 5e-5
ELEMENT_KEYS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
                "start_ns", "end_ns")

pytestmark = pytest.mark.gpu


def fixture():
    g = np.load(GOLDEN / "order0_c0.npz")
    el = {k: g[k] for k in ELEMENT_KEYS}
    return g, el


def optics_of(g, order=8):
    from lighthit_b200.order0 import Order0Optics
    return Order0Optics.from_arrays(g, order=order)


def oracle_args(g):
    det = dict(positions_m=g["positions_m"], looks=g["looks"], areas_m2=g["areas_m2"],
               radii_m=g["radii_m"], alpha=g["alpha"])
    optics = {k: g[k] for k in ("panel_edges", "phase_nodes", "group_nodes", "extinction_nodes",
                                "efficiency_coefficients")}
    return det, optics


def check_against(q, b, q_ref, b_ref):
    big = np.abs(q_ref) > 1e-6
    assert np.all(q[~big] < 1e-5)
    rel = np.abs(q - q_ref)[big] / np.abs(q_ref)[big]
    assert rel.max() < ORDER0_CHARGE_TOL, rel.max()
    if b is not None:
        l1 = np.abs(b - b_ref).sum(axis=1)[big] / np.abs(q_ref)[big]
        assert l1.max() < ORDER0_BINS_TOL, l1.max()


def test_device_bins_match_reference_rays_order8():
    from lighthit_b200.order0 import order0
    g, el = fixture()
    out = order0(optics_of(g), [el], g["origins_ns"][None], g["edges_ns"])
    q = out["charge"][0].cpu().numpy()
    b = out["bins"][0].cpu().numpy()
    check_against(q, b, g["rays8_charge"], g["rays8_bins"])
    # every bin sum is the charge (one quadrature)
    assert np.abs(b.sum(axis=1) - q).max() <= 1e-12 * q.max()


def test_device_charge_matches_route_order0():
    """Charge only (edges +-1e100) against the route's own control-variate order 0."""
    from lighthit_b200.order0 import order0
    g, el = fixture()
    s = np.load(GOLDEN / "shower_c0.npz")
    out = order0(optics_of(g), [el])
    q = out["charge"][0].cpu().numpy()
    ref = s["charge_components_pe"][:, 0]
    big = ref > 1e-3
    assert (np.abs(q[big] - ref[big]) / ref[big]).max() < ORDER0_CHARGE_TOL


def test_device_order16_matches_oracle_subset():
    from lighthit_b200.order0 import order0
    g, el = fixture()
    det, optics = oracle_args(g)
    sub = g["sub_pairs"]
    # the oracle on a pair subset: restrict the elements to the subset's elements
    keep = np.unique(g["pair_element"][sub])
    el_sub = {k: v[keep] for k, v in el.items()}
    po, pe = oracle.candidates(g["positions_m"], g["radii_m"], el_sub["start_m"],
                               el_sub["direction"], el_sub["length_m"], el_sub["coefficient0"],
                               el_sub["beta"], g["phase_nodes"])
    q_ref, b_ref = oracle.rays(po, pe, det, el_sub, optics, g["origins_ns"], g["edges_ns"], 16)
    out = order0(optics_of(g, 16), [el_sub], g["origins_ns"][None], g["edges_ns"])
    check_against(out["charge"][0].cpu().numpy(), out["bins"][0].cpu().numpy(), q_ref, b_ref)


def test_batched_events_equal_alone_and_ragged():
    """Several events of uneven size (one empty of light) in one launch."""
    from lighthit_b200.order0 import order0
    g, el = fixture()
    opt = optics_of(g)
    rng = np.random.default_rng(5)
    events = []
    for size in (1, 37, 700, 2000):
        pick = np.sort(rng.choice(len(el["beta"]), size, replace=False))
        events.append({k: v[pick] for k, v in el.items()})
    origins = np.repeat(g["origins_ns"][None], len(events), axis=0)
    both = order0(opt, events, origins, g["edges_ns"])
    for k, ev in enumerate(events):
        alone = order0(opt, [ev], origins[:1], g["edges_ns"])
        qa, qb = alone["charge"][0].cpu().numpy(), both["charge"][k].cpu().numpy()
        assert np.abs(qa - qb).max() <= 1e-12 * max(qa.max(), 1e-30)
        ba, bb = alone["bins"][0].cpu().numpy(), both["bins"][k].cpu().numpy()
        assert np.abs(ba - bb).max() <= 1e-12 * max(ba.max(), 1e-30)
    # the 2000-element draw is the whole set: the fixture's rays
    check_against(both["charge"][3].cpu().numpy(), both["bins"][3].cpu().numpy(),
                  g["rays8_charge"], g["rays8_bins"])


def test_fine_bins_and_shifted_clock_vs_oracle():
    """1 ns bins over a shifted window on a subset (many s and phi cuts)."""
    from lighthit_b200.order0 import order0
    g, el = fixture()
    det, optics = oracle_args(g)
    keep = np.arange(0, len(el["beta"]), 7)
    el_sub = {k: v[keep] for k, v in el.items()}
    po, pe = oracle.candidates(g["positions_m"], g["radii_m"], el_sub["start_m"],
                               el_sub["direction"], el_sub["length_m"], el_sub["coefficient0"],
                               el_sub["beta"], g["phase_nodes"])
    edges = np.arange(-60.0, 2001.0, 1.0)
    origins = g["origins_ns"] - 3.3
    q_ref, b_ref = oracle.rays(po, pe, det, el_sub, optics, origins, edges, 8)
    out = order0(optics_of(g), [el_sub], origins[None], edges)
    check_against(out["charge"][0].cpu().numpy(), out["bins"][0].cpu().numpy(), q_ref, b_ref)


def test_segment_through_glass_raises_like_reference():
    from lighthit_b200.order0 import order0
    g, el = fixture()
    el2 = {k: np.array(v, copy=True) for k, v in el.items()}
    i, om = int(g["pair_element"][0]), int(g["pair_om"][0])
    el2["start_m"][i] = g["positions_m"][om] - el2["direction"][i] * 0.05
    with pytest.raises(ValueError, match="intersects the glass"):
        order0(optics_of(g), [el2])
