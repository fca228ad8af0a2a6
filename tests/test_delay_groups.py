"""``delay_groups`` (``shower/ge2.py:122-147``) on the host, against the reference (CPU).

The delayed-light fixture (``tests/golden/make_shower_delayed_golden.py``)
holds the reference route's split of the README shower plus delayed copies:
groups inside the readout window and steps beyond it. The host split of the
device route must give the same groups and counts.
"""
import numpy as np

from conftest import GOLDEN

FIELDS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
          "start_ns", "end_ns")


def test_delay_groups_match_the_reference_split():
    from lighthit_b200.shower import ShowerSettings, delay_groups
    g = np.load(GOLDEN / "shower_delayed_c0.npz")
    route = np.load(GOLDEN.parent.parent / "lighthit_b200" / "tables" / "route_c0.npz")
    el = np.load(GOLDEN / "order0_c0.npz")
    base = {k: np.asarray(el[k], float) for k in FIELDS}
    parts = [np.arange(len(base["beta"])), g["delayed_a"], g["beyond"]]
    delays = [0.0, *[float(d) for d in g["delays"]]]
    source = {k: np.concatenate([base[k][idx] + (d if k.endswith("_ns") else 0.0)
                                 for idx, d in zip(parts, delays)]) for k in FIELDS}
    cfg = ShowerSettings()
    prompt, groups, beyond = delay_groups(
        source, prompt_delay_ns=cfg.prompt_delay_ns, cell_ns=cfg.delayed_cell_ns,
        window_end_ns=float(route["edges_ns"][-1]),
        group_index_max=float(np.max(route["group_index"])))
    assert len(groups) == int(g["groups_in_window"])
    assert int(beyond.sum()) == int(g["steps_beyond_window"])
    assert int(prompt.sum()) == len(base["beta"])
    assert sum(int(m.sum()) for m, _ in groups) == len(g["delayed_a"])
    assert all(shift > cfg.prompt_delay_ns for _, shift in groups)
    # every step is in exactly one of prompt, a group, beyond
    total = prompt.astype(int) + beyond.astype(int) + sum(m.astype(int) for m, _ in groups)
    assert np.all(total == 1)
