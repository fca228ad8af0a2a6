"""Order >=2 contraction: oracle pinned to the reference, device kernel vs oracle."""
import numpy as np
import pytest

from conftest import GOLDEN, TABLES
from oracle.ge2 import apply_folded as oracle_apply

# Device >=2 spectra: float32 contraction, float64 geometry. Error relative to
# the largest |value| of the spectrum (>=2 charges can be slightly negative).
GE2_TOL = 2e-5


def fixture():
    g = np.load(GOLDEN / "shower_c0.npz")
    t = dict(np.load(TABLES / "ge2_fold_48om_2-150m.npz"))
    frame = dict(centre=g["frame_centre_m"], first=g["frame_first"], second=g["frame_second"],
                 axis=g["frame_axis"])
    return g, t, frame


def points(g, frame, tag):
    z, tr = g[f"{tag}_z_m"], g[f"{tag}_transverse_m"]
    return (frame["centre"][None] + z[:, None] * frame["axis"][None]
            + tr[:, 0:1] * frame["first"][None] + tr[:, 1:2] * frame["second"][None])


def oracle_sources(g, frame, tag, channels=None):
    return dict(points_m=points(g, frame, tag),
                channels=g[f"{tag}_channels"] if channels is None else channels,
                reference_ns=g[f"{tag}_reference_ns"], frame=frame,
                degree=int(g["source_degree"]), azimuthal_degree=int(g["azimuthal_degree"]))


def test_oracle_matches_reference_full_frequency_subset():
    g, t, frame = fixture()
    out = oracle_apply(t, oracle_sources(g, frame, "sub"), g["om_positions_m"], g["om_looks"],
                       g["alpha"], g["om_area_m2"], g["radial_window_m"])
    assert np.abs(out - g["spec_sub"]).max() <= 1e-12 * np.abs(g["spec_sub"]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["zero", "sub"])
def test_device_apply_matches_reference(tag):
    from lighthit_b200.ge2 import AxialSources, Ge2Table
    g, t, frame = fixture()
    table = Ge2Table(t, g["alpha"], source_degree=int(g["source_degree"]),
                     azimuthal_degree=int(g["azimuthal_degree"]))
    src = AxialSources(points(g, frame, tag), g[f"{tag}_channels"], g[f"{tag}_reference_ns"],
                       (frame["centre"], frame["first"], frame["second"], frame["axis"]),
                       int(g["source_degree"]), int(g["azimuthal_degree"]))
    out = table.apply(src, g["om_positions_m"], g["om_looks"], g["om_area_m2"],
                      g["radial_window_m"], zero_frequency=(tag == "zero"))
    ref = g[f"spec_{tag}"]
    assert out.shape == ref.shape
    assert np.abs(out - ref).max() <= GE2_TOL * np.abs(ref).max()


@pytest.mark.gpu
def test_device_apply_all_points_random_channels_vs_oracle():
    """Every basis point at all 65 frequencies (seeded channels), vs the oracle."""
    from lighthit_b200.ge2 import AxialSources, Ge2Table
    g, t, frame = fixture()
    rng = np.random.default_rng(8)
    P = int(g["n_points"])
    zero_pts = points(g, frame, "zero")
    ch = (rng.normal(size=(3, P, 39, 65)) + 1j * rng.normal(size=(3, P, 39, 65))).astype(np.complex64)
    ch *= np.abs(g["zero_channels"][:, :, :, :1])  # keep the sources' magnitude profile
    oms = np.arange(0, 48, 4)
    src_o = dict(points_m=zero_pts, channels=ch, reference_ns=np.array([0.0, 0.3, -0.2]),
                 frame=frame, degree=int(g["source_degree"]),
                 azimuthal_degree=int(g["azimuthal_degree"]))
    ref = oracle_apply(t, src_o, g["om_positions_m"][oms], g["om_looks"][oms], g["alpha"],
                       g["om_area_m2"][oms], g["radial_window_m"])
    table = Ge2Table(t, g["alpha"], source_degree=8, azimuthal_degree=2)
    src = AxialSources(zero_pts, ch, src_o["reference_ns"],
                       (frame["centre"], frame["first"], frame["second"], frame["axis"]), 8, 2)
    out = table.apply(src, g["om_positions_m"][oms], g["om_looks"][oms], g["om_area_m2"][oms],
                      g["radial_window_m"])
    assert np.abs(out - ref).max() <= GE2_TOL * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("zero_frequency", [True, False])
def test_batched_problems_equal_alone(zero_frequency):
    """Problems of one batched launch (different OM subsets, sources, frames,
    one without points) equal each problem applied alone, bit for bit: the
    point chunks are summed in the same fixed order either way."""
    from lighthit_b200.ge2 import AxialSources, Ge2Table
    g, t, frame = fixture()
    table = Ge2Table(t, g["alpha"], source_degree=8, azimuthal_degree=2)
    rng = np.random.default_rng(17)
    pts = points(g, frame, "zero")
    P = len(pts)
    basis = (frame["centre"], frame["first"], frame["second"], frame["axis"])
    items = []
    for k, oms in enumerate([np.arange(48), np.arange(3, 40, 5), np.array([7])]):
        ch = (rng.normal(size=(3, P, 39, 65)) + 1j * rng.normal(size=(3, P, 39, 65))).astype(
            np.complex64) * np.abs(g["zero_channels"][:, :, :, :1])
        shifted = tuple(np.asarray(v) + (0.3 * k * frame["axis"] if i == 0 else 0)
                        for i, v in enumerate(basis))
        src = AxialSources(pts + 0.3 * k * frame["axis"], ch, np.array([0.0, 0.1 * k, 0.0]),
                           shifted, 8, 2)
        items.append((src, g["om_positions_m"][oms], g["om_looks"][oms], g["om_area_m2"][oms],
                      g["radial_window_m"]))
    empty = AxialSources(np.zeros((0, 3)), np.zeros((3, 0, 39, 65), np.complex64),
                         np.zeros(3), basis, 8, 2)
    items.append((empty,) + items[1][1:])
    together = [r.cpu().numpy() for r in table.apply_batch(items, zero_frequency=zero_frequency)]
    for it, got in zip(items, together):
        alone = table.apply_device(*it, zero_frequency=zero_frequency).cpu().numpy()
        assert got.shape == alone.shape
        assert np.array_equal(got, alone)
    assert not np.any(together[-1])
    assert np.any(together[0])


# Tensor-core contraction: BF16 operands with float32 accumulation. Split-BF16
# carries 24 significant bits per operand (hi + mid + lo, six products), as the
# float32 contraction; a single BF16 product 8 bits. Error relative to the
# largest |value|.
TC_TOL = {"split-bf16": GE2_TOL, "bf16": 2e-2}


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["split-bf16", "bf16"])
def test_tensor_core_apply_vs_oracle(mode):
    """Every basis point at all 65 frequencies (seeded channels) through the
    tcgen05 contraction, against the float64 oracle and the float32 CUDA-core
    contraction."""
    from lighthit_b200.ge2 import AxialSources, Ge2Table
    g, t, frame = fixture()
    rng = np.random.default_rng(9)
    P = int(g["n_points"])
    pts = points(g, frame, "zero")
    ch = (rng.normal(size=(3, P, 39, 65)) + 1j * rng.normal(size=(3, P, 39, 65))).astype(np.complex64)
    ch *= np.abs(g["zero_channels"][:, :, :, :1])
    oms = np.arange(48)
    refs = np.array([0.0, 0.2, -0.1])
    src_o = dict(points_m=pts, channels=ch, reference_ns=refs, frame=frame,
                 degree=int(g["source_degree"]), azimuthal_degree=int(g["azimuthal_degree"]))
    ref = oracle_apply(t, src_o, g["om_positions_m"], g["om_looks"], g["alpha"],
                       g["om_area_m2"], g["radial_window_m"])
    table = Ge2Table(t, g["alpha"], source_degree=8, azimuthal_degree=2)
    assert table.tc_packed() is not None
    src = AxialSources(pts, ch, refs, (frame["centre"], frame["first"], frame["second"],
                                       frame["axis"]), 8, 2)
    item = (src, g["om_positions_m"][oms], g["om_looks"][oms], g["om_area_m2"][oms],
            g["radial_window_m"])
    out = table.apply_batch([item], mode=mode)[0].cpu().numpy().T
    assert int(table.status.item()) == 0
    fp32 = table.apply_batch([item], mode="fp32")[0].cpu().numpy().T
    scale = np.abs(ref).max()
    err, err32 = np.abs(out - ref).max() / scale, np.abs(fp32 - ref).max() / scale
    print(f"\n{mode}: max error {err:.2e} of the largest value (fp32 CUDA cores {err32:.2e})")
    assert err <= TC_TOL[mode]


@pytest.mark.gpu
def test_tensor_core_batched_problems_equal_alone():
    """The tensor-core path computes every (OM, point) pair on its own and sums
    the points in a fixed order: a problem's spectrum is the same bit for bit
    alone and in a batch (other OMs, sources, frames, an empty problem)."""
    from lighthit_b200.ge2 import AxialSources, Ge2Table
    g, t, frame = fixture()
    table = Ge2Table(t, g["alpha"], source_degree=8, azimuthal_degree=2)
    rng = np.random.default_rng(18)
    pts = points(g, frame, "zero")
    P = len(pts)
    basis = (frame["centre"], frame["first"], frame["second"], frame["axis"])
    items = []
    for k, oms in enumerate([np.arange(48), np.arange(3, 40, 5), np.array([7])]):
        ch = (rng.normal(size=(3, P, 39, 65)) + 1j * rng.normal(size=(3, P, 39, 65))).astype(
            np.complex64) * np.abs(g["zero_channels"][:, :, :, :1])
        shifted = tuple(np.asarray(v) + (0.3 * k * frame["axis"] if i == 0 else 0)
                        for i, v in enumerate(basis))
        src = AxialSources(pts + 0.3 * k * frame["axis"], ch, np.array([0.0, 0.1 * k, 0.0]),
                           shifted, 8, 2)
        items.append((src, g["om_positions_m"][oms], g["om_looks"][oms], g["om_area_m2"][oms],
                      g["radial_window_m"]))
    empty = AxialSources(np.zeros((0, 3)), np.zeros((3, 0, 39, 65), np.complex64),
                         np.zeros(3), basis, 8, 2)
    items.append((empty,) + items[1][1:])
    together = [r.cpu().numpy() for r in table.apply_batch(items, mode="split-bf16")]
    assert int(table.status.item()) == 0
    for it, got in zip(items, together):
        alone = table.apply_batch([it], mode="split-bf16")[0].cpu().numpy()
        assert np.array_equal(got, alone)
    assert not np.any(together[-1])
    assert np.any(together[0])
