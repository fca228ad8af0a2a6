"""Order 1 (grouped pencils) on the device against the reference's fixtures (``-m gpu``).

Fixtures: ``tests/golden/order1_c0.npz`` (``make_order1_golden.py``), the
README-example shower with the shower route's prompt settings.

Tolerances. The device sums moments with float64 atomics (order differs from
the reference's sequential sums, ~1e-15 relative); a pencil or group whose
key sits on a cell, pixel, tau, log-r or theta boundary can land on the other
side, which moves that pencil's light between neighbouring groups: the
grouped result then differs by that group's share of the grouping error. The
per-OM charge agrees to ORDER1_CHARGE_TOL relative (OMs above 1e-4 pe) and
the bins to ORDER1_BINS_TOL of the OM's charge (L1).
"""
import numpy as np
import pytest

from conftest import GOLDEN

ORDER1_CHARGE_TOL = 1e-6
ORDER1_BINS_TOL = 1e-5
PENCIL_KEYS = ("position", "direction", "w0", "w2", "time", "major", "var_major", "var_minor",
               "pos_cov")
ELEMENT_KEYS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
                "start_ns", "end_ns")

pytestmark = pytest.mark.gpu


def fixture():
    return np.load(GOLDEN / "order1_c0.npz")


def tables_of(g):
    from lighthit_b200.order1 import Order1Tables, PromptSettings
    settings = PromptSettings(
        cell_m=float(g["cell_m"]), pixel_face=int(g["pixel_face"]),
        ring_nodes=int(g["ring_nodes"]), path_step=float(g["path_step"]),
        path_step_tail=float(g["path_step_tail"]), tail_exponent=float(g["tail_exponent"]),
        direct_bins=int(g["direct_bins"]), max_path_nodes=int(g["max_path_nodes"]),
        smoothing_factor=float(g["smoothing_factor"]),
        merge_theta_min=float(g["merge_theta_min"]),
        merge_theta_ratio=float(g["merge_theta_ratio"]), merge_tau_ns=float(g["merge_tau_ns"]),
        merge_log_r=float(g["merge_log_r"]))
    bands = {k: g[k] for k in ("mus", "mut", "speed", "s0w", "s2w")}
    mono = (g["coef"], g["ipow"], g["jpow"], int(g["degree"]))
    return Order1Tables(bands, float(g["g"]), mono, g["positions_m"], g["looks"], g["areas_m2"],
                        g["edges_ns"], settings=settings)


def check(q, b, q_ref, b_ref):
    big = np.abs(q_ref) > 1e-4
    rel = np.abs(q - q_ref)[big] / np.abs(q_ref)[big]
    assert rel.max() < ORDER1_CHARGE_TOL, rel.max()
    assert np.abs(q - q_ref)[~big].max(initial=0.0) < 1e-4 * ORDER1_CHARGE_TOL * 1e4
    l1 = np.abs(b - b_ref).sum(axis=1)[big] / np.abs(q_ref)[big]
    assert l1.max() < ORDER1_BINS_TOL, l1.max()


def test_grouped_on_reference_pencils():
    """Stage B alone: the reference's own pencils of a 64-element subset, all OMs."""
    from lighthit_b200.order1 import PencilTable, grouped
    g = fixture()
    tables = tables_of(g)
    pencils = {k: g[f"sub_pencil_{k}"] for k in PENCIL_KEYS}
    table, n = PencilTable.from_host(pencils, tables.device)
    q, b = grouped(tables, table, np.arange(tables.n_om), g["origins_ns"], n_pencils=n)
    check(q.cpu().numpy(), b.cpu().numpy(), g["sub_charge"], g["sub_bins"])


def test_pencils_match_reference_compress():
    """Stage A alone: the pencil table of the 64-element subset, as a set of rows."""
    from lighthit_b200.order1 import pencils
    g = fixture()
    tables = tables_of(g)
    pick = g["sub_pick"]
    el = {k: g[k][pick] for k in ELEMENT_KEYS}
    table = pencils(tables, el, g["cone_cos"][pick])
    got = table.host()
    ref = {k: g[f"sub_pencil_{k}"] for k in PENCIL_KEYS}
    assert len(got["w0"]) == len(ref["w0"])

    def order(p):
        return np.lexsort((np.round(p["direction"][:, 2], 9), np.round(p["direction"][:, 1], 9),
                           np.round(p["direction"][:, 0], 9), np.round(p["position"][:, 2], 9),
                           np.round(p["position"][:, 1], 9), np.round(p["position"][:, 0], 9)))
    a, r = order(got), order(ref)
    for k in PENCIL_KEYS:
        x, y = got[k][a], ref[k][r]
        scale = max(np.abs(y).max(), 1e-300)
        assert np.abs(x - y).max() <= 1e-9 * scale, k


def test_fine_order1_all_elements_matches_reference():
    """Stages A + B on all 2000 elements: the fine order 1 of every OM."""
    from lighthit_b200.order1 import order1
    g = fixture()
    tables = tables_of(g)
    el = {k: g[k] for k in ELEMENT_KEYS}
    q, b = order1(tables, el, g["cone_cos"], g["origins_ns"])
    check(q.cpu().numpy(), b.cpu().numpy(), g["full_charge"], g["full_bins"])


def test_work_subset_leaves_other_oms_zero():
    from lighthit_b200.order1 import PencilTable, grouped
    g = fixture()
    tables = tables_of(g)
    pencils = {k: g[f"sub_pencil_{k}"] for k in PENCIL_KEYS}
    table, n = PencilTable.from_host(pencils, tables.device)
    work = np.array([3, 17, 40])
    q, b = grouped(tables, table, work, g["origins_ns"], n_pencils=n)
    q, b = q.cpu().numpy(), b.cpu().numpy()
    rest = np.setdiff1d(np.arange(tables.n_om), work)
    assert np.all(q[rest] == 0) and np.all(b[rest] == 0)
    check(q[work], b[work], g["sub_charge"][work], g["sub_bins"][work])


def test_screen_pack_matches_oracle():
    """The coarse screen's stage A on the device: parents (8-pixel faces) and
    children (32-pixel faces) equal the oracle's pack (compress_screen,
    _prompt_screen.py:56-98), each child pointing at its own parent."""
    from lighthit_b200.order1 import Order1Tables, PromptSettings, pencils
    from oracle import order1 as O1
    g = np.load(GOLDEN / "order1_c0.npz")
    el = {k: g[k] for k in ("start_m", "direction", "length_m", "coefficient0", "coefficient2",
                            "beta", "start_ns", "end_ns")}
    tables = Order1Tables({k: g[k] for k in ("mus", "mut", "speed", "s0w", "s2w")},
                          float(g["g"]), (g["coef"], g["ipow"], g["jpow"], int(g["degree"])),
                          g["positions_m"], g["looks"], g["areas_m2"], g["edges_ns"],
                          settings=PromptSettings().coarse(), compute_bins=False)
    table = pencils(tables, el, g["cone_cos"])
    n = int(table.count.item())
    dev = {k: v[:n].cpu().numpy() for k, v in table.t.items()}
    parent = table.parent[:n].cpu().numpy()
    ref = O1.screen_pencils(el, g["cone_cos"])
    roots = parent < 0
    assert n == len(ref["w0"]) and roots.sum() == (ref["hierarchy_parent"] == -2).sum()
    for mask_dev, mask_ref in ((roots, ref["hierarchy_parent"] == -2),
                               (~roots, ref["hierarchy_parent"] >= 0)):
        a = np.sort(dev["w0"][mask_dev])
        b = np.sort(ref["w0"][mask_ref])
        assert np.abs(a - b).max() <= 1e-12 * b.max()
    # every child's parent carries its weight: parents equal their children's sums
    sums = np.bincount(parent[~roots], weights=dev["w0"][~roots], minlength=n)
    assert np.allclose(sums[roots], dev["w0"][roots], rtol=1e-12, atol=0)
    assert np.all(roots[parent[~roots]])


@pytest.mark.parametrize("step", [0.01, 0.004])
def test_long_path_grids_match_the_oracle(step):
    """Path steps 10 and 25 times finer than the route's (typical grids of
    ~330 and ~830 nodes against ~33): grids past the 512 nodes that the small
    batch instance holds in shared memory are handed to the full-size
    instance. Stage B on the reference's pencils against the oracle's grouped
    order 1 with the same steps (the finer grids move the charge by ~2e-5, so
    the comparison sees the grid)."""
    from dataclasses import replace
    from lighthit_b200.order1 import Order1Tables, PencilTable, grouped
    from oracle import order1 as O1
    g = fixture()
    base = tables_of(g)
    s = replace(base.settings, path_step=step, path_step_tail=2.5 * step)
    tables = Order1Tables({k: g[k] for k in ("mus", "mut", "speed", "s0w", "s2w")},
                          float(g["g"]), (g["coef"], g["ipow"], g["jpow"], int(g["degree"])),
                          g["positions_m"], g["looks"], g["areas_m2"], g["edges_ns"], settings=s)
    pencils = {k: g[f"sub_pencil_{k}"] for k in PENCIL_KEYS}
    table, n = PencilTable.from_host(pencils, tables.device)
    work = np.arange(tables.n_om)
    q, b = grouped(tables, table, work, g["origins_ns"], n_pencils=n)
    q_ref, b_ref, _, _ = O1.grouped(
        pencils, g["positions_m"], g["looks"], g["areas_m2"], g["origins_ns"], work,
        (g["coef"], g["ipow"], g["jpow"], int(g["degree"])), float(g["g"]),
        {k: g[k] for k in ("mus", "mut", "speed", "s0w", "s2w")}, g["edges_ns"],
        path_step=step, path_step_tail=2.5 * step, tail_exponent=float(g["tail_exponent"]),
        direct_bins=int(g["direct_bins"]), max_path_nodes=int(g["max_path_nodes"]),
        smoothing_factor=float(g["smoothing_factor"]),
        merge=(float(g["merge_theta_min"]), float(g["merge_theta_ratio"]),
               float(g["merge_tau_ns"]), float(g["merge_log_r"])))
    check(q.cpu().numpy(), b.cpu().numpy(), q_ref, b_ref)
