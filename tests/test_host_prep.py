"""Host-side operator construction (float64, no GPU)."""
import numpy as np
import pytest
from scipy.interpolate import CubicSpline

from conftest import GOLDEN, TABLES
from lighthit_b200.readout import readout_matrix
from lighthit_b200.spline import resample_matrix, spline_coefficients


@pytest.mark.parametrize("n", [4, 7, 48, 65])
def test_spline_coefficients_match_scipy(n):
    rng = np.random.default_rng(n)
    x = np.sort(rng.uniform(0, 3, n)) + np.arange(n) * 0.05
    y = rng.normal(size=(n, 3)) + 1j * rng.normal(size=(n, 3))
    c = spline_coefficients(x, y, axis=0)  # (n-1, 4, 3)
    ref = CubicSpline(x, y.real, axis=0).c + 1j * CubicSpline(x, y.imag, axis=0).c
    scale = np.abs(ref).max()
    assert np.max(np.abs(np.moveaxis(c, 1, 0) - ref)) < 1e-11 * scale


def test_resample_matrix_matches_scipy():
    o = np.linspace(0, 1.2, 65)
    o2 = np.linspace(0, 1.2, 321)
    y = np.random.default_rng(1).normal(size=(65, 4))
    assert np.max(np.abs(resample_matrix(o, o2) @ y - CubicSpline(o, y, axis=0)(o2))) < 1e-13


def test_readout_matrix_matches_reference_fixture():
    g = np.load(GOLDEN / "readout_c0.npz")
    W = readout_matrix(g["omega_per_ns"], g["edges_ns"], g["readout_omega_per_ns"])
    assert np.max(np.abs((W @ g["relative"]).real.T - g["bins"])) < 1e-13


def test_flash_spline_table_reproduces_oracle_moments(flash_table):
    from oracle.flash import moments_at
    t = flash_table
    table = dict(np.load(TABLES / "flash_450nm_2-250m.npz"))
    coef = t.spline_table(2)  # (j, w, l, o, p)
    r = np.array([2.0, 3.3, 17.0, 99.9, 200.0, 250.0])
    log_r = np.log(t.radii_m)
    j = np.clip(np.searchsorted(log_r, np.log(r), side="right") - 1, 0, len(log_r) - 2)
    tt = np.log(r) - log_r[j]
    c = coef[j]  # (n, w, l, o, p)
    val = ((c[..., 0] * tt[:, None, None, None] + c[..., 1]) * tt[:, None, None, None]
           + c[..., 2]) * tt[:, None, None, None] + c[..., 3]
    scale = np.exp(-t.medium.absorption_per_m * r) / (4 * np.pi * r ** 2)
    flight = np.exp(1j * t.omega_per_ns[None, :] * r[:, None] / t.medium.speed_m_per_ns)
    got = val * scale[:, None, None, None] * flight[:, :, None, None]  # (n, w, l, o)
    ref = moments_at(table, r, 3)  # (w, n, l, o)
    ref = np.moveaxis(ref, 1, 0)
    assert np.max(np.abs(got - ref)) < 1e-9 * np.abs(ref).max()


def test_acceptance_coefficients_match_fixture(flash_golden):
    from lighthit_b200.model import acceptance_coefficients, synthetic_detector
    det = synthetic_detector()
    alpha = acceptance_coefficients(det.angular_acceptance, 8)
    assert np.max(np.abs(alpha - flash_golden["alpha"])) < 1e-11
    np.testing.assert_array_equal(det.positions_m, flash_golden["om_positions_m"])


def test_axis_frame_is_bit_identical_to_the_reference_expressions():
    """``axis_frame`` reproduces ``AxisFrame.of`` (``axial_source.py:88-118``) bit for
    bit: its running sums equal NumPy's ``sum(axis=0)`` and three-operand ``einsum``."""
    from lighthit_b200.source import axis_frame
    rng = np.random.default_rng(5)
    for n in (1, 7, 2000, 50000):
        start = rng.normal(size=(n, 3)) * 30
        direction = rng.normal(size=(n, 3))
        direction /= np.linalg.norm(direction, axis=1)[:, None]
        length = rng.uniform(0.01, 2.0, n)
        weights = rng.uniform(0.1, 3.0, n)
        points = start + 0.5 * length[:, None] * direction
        share = weights / weights.sum()
        centre = (share[:, None] * points).sum(axis=0)
        offset = points - centre
        covariance = np.einsum("i,ij,ik->jk", share, offset, offset)
        values, vectors = np.linalg.eigh(covariance)
        got = axis_frame(start, direction, length, weights)
        assert np.array_equal(got[0], centre)
        if n > 1:
            axis = vectors[:, int(np.argmax(values))]
            axis = axis / np.linalg.norm(axis)
            if float((share * (direction @ axis)).sum()) < 0:
                axis = -axis
            assert np.array_equal(got[1], axis)


def _steps(n, seed):
    rng = np.random.default_rng(seed)
    direction = rng.normal(size=(n, 3))
    direction /= np.linalg.norm(direction, axis=1)[:, None]
    return (rng.normal(scale=30.0, size=(n, 3)), direction, rng.uniform(0.0, 0.3, n),
            rng.uniform(0.0, 200.0, n))


@pytest.mark.parametrize("n", [1, 7, 5000])
def test_element_box_is_the_numpy_box(n):
    from lighthit_b200.order1 import element_box
    start, direction, length, _ = _steps(n, n)
    ends = start + length[:, None] * direction
    low, high = element_box({"start_m": start, "direction": direction, "length_m": length})
    assert np.array_equal(low, np.minimum(start.min(axis=0), ends.min(axis=0)))
    assert np.array_equal(high, np.maximum(start.max(axis=0), ends.max(axis=0)))
    start[n // 2, 1] = np.nan  # NaN bounds for that coordinate only, as NumPy
    low, high = element_box({"start_m": start, "direction": direction, "length_m": length})
    assert np.isnan(low[1]) and np.isnan(high[1]) and np.isfinite(low[[0, 2]]).all()


def test_delay_groups_match_the_numpy_expressions():
    from lighthit_b200.shower import C_M_PER_NS, delay_groups
    start, direction, length, t0 = _steps(4000, 5)
    el = {"start_m": start, "direction": direction, "length_m": length, "start_ns": t0}
    first = int(np.argmin(t0))
    d0 = start - start[first]
    distance = np.sqrt(d0[:, 0] * d0[:, 0] + d0[:, 1] * d0[:, 1] + d0[:, 2] * d0[:, 2])
    delay = t0 - t0[first] - distance / C_M_PER_NS
    kw = dict(prompt_delay_ns=20.0, cell_ns=10.0, window_end_ns=100.0, group_index_max=1.4)
    prompt, groups, beyond = delay_groups(el, **kw)
    assert np.array_equal(prompt, delay <= 20.0)
    far = ~prompt & (delay - 0.4 * distance / C_M_PER_NS > 100.0)
    assert np.array_equal(beyond, far)
    within = ~prompt & ~far
    cells = np.floor(delay / 10.0).astype(np.int64)
    expected = [(within & (cells == c), float(delay[within & (cells == c)].min()))
                for c in np.unique(cells[within])]
    assert len(groups) == len(expected) > 1
    for (m, shift), (m_ref, shift_ref) in zip(groups, expected):
        assert np.array_equal(m, m_ref) and shift == shift_ref


def test_subsegment_offsets_are_the_numpy_running_totals():
    from lighthit_b200 import _lib
    rng = np.random.default_rng(9)
    length = np.ascontiguousarray(np.concatenate([rng.uniform(0.0, 3.0, 4000), [0.0, 0.25, 0.5]]))
    step = 0.25
    expected = np.zeros(len(length) + 1, np.int64)
    expected[1:] = np.cumsum(np.maximum(1, np.ceil(length / step)).astype(np.int64))
    offsets, total = np.empty(len(length) + 1, np.int64), np.zeros(1, np.int64)
    lib = _lib.load()
    assert lib.lh_subsegment_offsets(len(length), length.ctypes.data, step, offsets.ctypes.data,
                                     total.ctypes.data) == 0
    assert np.array_equal(offsets, expected) and total[0] == expected[-1]
    bad = np.array([1.0, np.nan])
    assert lib.lh_subsegment_offsets(2, bad.ctypes.data, step, offsets.ctypes.data,
                                     total.ctypes.data) != 0
