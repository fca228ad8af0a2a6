"""The CPU oracle of the shower route, pinned to the reference's own outputs.

The fixtures were written by the reference's float64 route
(``tests/golden/make_*_golden.py``): stage-A pencils and grouped order 1 of
the README shower (``order1_c0.npz``), its node-band sources
(``source_c0.npz``) and >=2 spectra and full response (``shower_c0.npz``),
and full responses of the seeded config-2 stream (``shower_c2.npz``).
"""
import numpy as np
import pytest

from conftest import GOLDEN, TABLES

ELEMENT_KEYS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
                "start_ns", "end_ns")


def test_order1_stage_a_and_b_bit_identical():
    from oracle import order1 as O1
    g = np.load(GOLDEN / "order1_c0.npz")
    el = {k: g[k] for k in ELEMENT_KEYS}
    kw = dict(cell_m=float(g["cell_m"]), pixel_face=int(g["pixel_face"]),
              ring_nodes=int(g["ring_nodes"]))
    pick = g["sub_pick"]
    pen = O1.compress({k: v[pick] for k, v in el.items()}, g["cone_cos"][pick], **kw)
    for k, _ in O1.FIELDS:
        np.testing.assert_array_equal(pen[k], g["sub_pencil_" + k])
    mono = (g["coef"], g["ipow"], g["jpow"], int(g["degree"]))
    bands = {k: g[k] for k in ("mus", "mut", "speed", "s0w", "s2w")}
    settings = dict(path_step=float(g["path_step"]), path_step_tail=float(g["path_step_tail"]),
                    tail_exponent=float(g["tail_exponent"]), direct_bins=int(g["direct_bins"]),
                    max_path_nodes=int(g["max_path_nodes"]),
                    smoothing_factor=float(g["smoothing_factor"]),
                    merge=(float(g["merge_theta_min"]), float(g["merge_theta_ratio"]),
                           float(g["merge_tau_ns"]), float(g["merge_log_r"])))
    args = (g["positions_m"], g["looks"], g["areas_m2"], g["origins_ns"], np.arange(48), mono,
            float(g["g"]), bands, g["edges_ns"])
    q, b, groups, batches = O1.grouped(pen, *args, **settings)
    np.testing.assert_array_equal(q, g["sub_charge"])
    np.testing.assert_array_equal(b, g["sub_bins"])
    np.testing.assert_array_equal(groups, g["sub_groups"])
    np.testing.assert_array_equal(batches, g["sub_batches"])
    full = O1.compress(el, g["cone_cos"], **kw)
    assert len(full["w0"]) == int(g["full_pencils"])
    q, b, groups, batches = O1.grouped(full, *args, **settings)
    np.testing.assert_array_equal(q, g["full_charge"])
    np.testing.assert_array_equal(b, g["full_bins"])
    np.testing.assert_array_equal(groups, g["full_groups"])


def test_screen_pack_is_a_preorder_hierarchy():
    """compress_screen's pack: every parent precedes its children, which carry
    its emission (pack_pencils, _prompt_screen.py:56-85)."""
    from oracle import order1 as O1
    g = np.load(GOLDEN / "order1_c0.npz")
    el = {k: g[k] for k in ELEMENT_KEYS}
    pack = O1.screen_pencils(el, g["cone_cos"])
    parent, nxt = pack["hierarchy_parent"], pack["next_node"]
    roots = np.flatnonzero(parent == -2)
    assert roots[0] == 0 and len(roots) < len(parent)
    for r, stop in zip(roots, np.r_[roots[1:], len(parent)]):
        assert nxt[r] == stop
        kids = np.arange(r + 1, stop)
        assert np.all(parent[kids] == r)
        assert pack["w0"][kids].sum() == pytest.approx(pack["w0"][r], rel=1e-12)


def test_source_oracle_matches_reference_node_sources():
    from oracle import source as S
    g = np.load(GOLDEN / "source_c0.npz")
    e = np.load(GOLDEN / "order0_c0.npz")
    el = {k: np.asarray(e[k], float) for k in ELEMENT_KEYS}
    frame = S.axis_frame(el, el["coefficient0"])
    for got, key in zip(frame, ("frame_centre_m", "frame_axis", "frame_first", "frame_second")):
        np.testing.assert_array_equal(got, g[key])
    sources = S.node_sources(el, g["wavelengths_nm"], g["phase_index"], g["scale"], g["bands"],
                             int(g["source_degree"]), int(g["azimuthal_degree"]),
                             g["omega_per_ns"], frame)
    for b, s in enumerate(sources):
        ref = g[f"band{b}_channels"]  # complex64 in the fixture
        np.testing.assert_array_equal(s.z_m, g[f"band{b}_z_m"])
        np.testing.assert_array_equal(s.transverse_m, g[f"band{b}_transverse_m"])
        assert np.abs(s.channels - ref).max() <= 2e-7 * np.abs(ref).max()
        assert s.reference_ns == float(g[f"band{b}_reference_ns"])


def test_ge2_c_loops_match_reference_spectra():
    from oracle.ge2 import apply_folded
    g = np.load(GOLDEN / "shower_c0.npz")
    t = dict(np.load(TABLES / "ge2_fold_48om_2-150m.npz"))
    frame = dict(centre=g["frame_centre_m"], first=g["frame_first"], second=g["frame_second"],
                 axis=g["frame_axis"])
    z, tr = g["sub_z_m"], g["sub_transverse_m"]
    pts = (frame["centre"][None] + z[:, None] * frame["axis"][None]
           + tr[:, 0:1] * frame["first"][None] + tr[:, 1:2] * frame["second"][None])
    src = dict(points_m=pts, channels=g["sub_channels"], reference_ns=g["sub_reference_ns"],
               frame=frame, degree=int(g["source_degree"]),
               azimuthal_degree=int(g["azimuthal_degree"]))
    out = apply_folded(t, src, g["om_positions_m"], g["om_looks"], g["alpha"], g["om_area_m2"],
                       g["radial_window_m"], fast=True)
    assert np.abs(out - g["spec_sub"]).max() <= 1e-12 * np.abs(g["spec_sub"]).max()


def check_route(out, charge, active, origins, components, threshold, *, charge_tol, bins_tol):
    q = out["charge_components_pe"]
    total = np.abs(charge.sum(axis=1))
    big = charge.sum(axis=1) >= threshold
    for o in range(3):
        assert (np.abs(q[big, o] - charge[big, o]) / total[big]).max(initial=0) <= charge_tol
    np.testing.assert_array_equal(out["active"], active)
    np.testing.assert_array_equal(out["time_origin_ns"], origins)
    both = active & out["active"]
    for o in range(3):
        l1 = np.abs(out["components_pe"][both, :, o] - components[both, :, o]).sum(axis=1)
        assert (l1 / np.maximum(total[both], 1e-30)).max(initial=0) <= bins_tol


def test_route_matches_reference_readme_shower():
    from oracle.shower import Route
    g = np.load(GOLDEN / "shower_c0.npz")
    e = np.load(GOLDEN / "order0_c0.npz")
    route = Route(np.load(TABLES / "route_c0.npz"), np.load(TABLES / "ge2_fold_48om_2-150m.npz"),
                  np.load(TABLES / "near_c0.npz"), order0_gauss=8, threads=4)
    out = route({k: e[k] for k in ELEMENT_KEYS})
    check_route(out, g["charge_components_pe"], g["active"], g["time_origin_ns"],
                g["components_pe"].astype(float), float(g["threshold_pe"]),
                charge_tol=1e-7, bins_tol=1e-5)
    np.testing.assert_array_equal(out["ge2_charge_level"], g["ge2_charge_level"])


@pytest.mark.parametrize("k", [6, 9])
def test_route_matches_reference_config2(k):
    from lighthit_b200.workloads import gaussian_shower, shower_stream
    from oracle.shower import Route
    g = np.load(GOLDEN / "shower_c2.npz")
    route = Route(np.load(TABLES / "route_c2.npz"), np.load(TABLES / "ge2_fold_384om_2-450m.npz"),
                  np.load(TABLES / "near_c2.npz"), order0_gauss=8, threads=4)
    s = shower_stream(k + 1, route.positions.mean(axis=0))[k]
    el = gaussian_shower(s["position_m"], s["direction"],
                         charged_track_length_m=s["charged_track_length_m"],
                         elements=s["elements"], seed=s["seed"])
    out = route(el)
    comp = np.zeros((len(route.positions), len(route.edges) - 1, 3))
    comp[g[f"s{k}_active_ids"]] = g[f"s{k}_components"]
    check_route(out, g[f"s{k}_charge"], g[f"s{k}_active"], g[f"s{k}_origin"], comp,
                float(route.threshold), charge_tol=1e-7, bins_tol=1e-5)
    # OMs the coarse screen left below threshold keep the screen's charge
    # (compress_screen / screen_order1 with the receiver-local refinement)
    coarse = out["prompt_order1_level"] == 1
    assert coarse.sum() > 100
    ref = g[f"s{k}_charge"][coarse, 1]
    got = out["charge_components_pe"][coarse, 1]
    assert (np.abs(got - ref) / np.maximum(np.abs(ref), 1e-12)).max() <= 1e-10
