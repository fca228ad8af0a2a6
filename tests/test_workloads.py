"""The seeded workload generators restate the reference's own draws."""
import numpy as np

from conftest import GOLDEN


def test_gaussian_shower_reproduces_reference_elements():
    """README-example shower (seed 7): the reference's SyntheticShower.gaussian elements."""
    from lighthit_b200.workloads import baikal_like_positions, gaussian_shower
    g = np.load(GOLDEN / "order0_c0.npz")
    positions, _ = baikal_like_positions(1)
    el = gaussian_shower(positions.mean(axis=0) + np.array([-12.0, 8.0, 0.0]),
                         [0.35, -0.15, 0.925], charged_track_length_m=300.0, elements=2000,
                         seed=7)
    for k, v in el.items():
        assert np.abs(v - g[k]).max() <= 1e-14 * max(np.abs(g[k]).max(), 1.0), k


def test_shower_stream_is_seeded_and_in_range():
    from lighthit_b200.workloads import shower_stream
    a = shower_stream(200, [630.0, 0.0, 0.0])
    b = shower_stream(200, [630.0, 0.0, 0.0])
    assert [x["elements"] for x in a] == [x["elements"] for x in b]
    n = np.array([x["elements"] for x in a])
    assert n.min() >= 500 and n.max() <= 50000
    pos = np.array([x["position_m"] for x in a]) - [630.0, 0.0, 0.0]
    assert np.all(np.hypot(pos[:, 0], pos[:, 1]) <= 200.0) and np.all(np.abs(pos[:, 2]) <= 300.0)
    d = np.array([x["direction"] for x in a])
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0)
