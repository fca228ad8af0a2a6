"""Order >=2 source compile on the device against the reference's fixture (``-m gpu``).

Fixture: ``tests/golden/source_c0.npz`` (``make_source_golden.py``): the
route's ``node_sources`` for the README-example shower on the rank-3 band fold.
Channels are stored as complex64 by both sides; per band they agree to
SOURCE_TOL of the band's largest channel, points to 1e-12 m.
"""
import numpy as np
import pytest

from conftest import GOLDEN

SOURCE_TOL = 2e-6
ELEMENT_KEYS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
                "start_ns", "end_ns")

pytestmark = pytest.mark.gpu


def compiled(frame_from_fixture=True):
    from lighthit_b200.source import ShowerBasisSettings, SourceCompiler
    g = np.load(GOLDEN / "source_c0.npz")
    el = np.load(GOLDEN / "order0_c0.npz")
    elements = {k: el[k] for k in ELEMENT_KEYS}
    settings = ShowerBasisSettings(cell_m=float(g["cell_m"]), stencil_m=float(g["stencil_m"]),
                                   stencil_threshold_m=float(g["stencil_threshold_m"]),
                                   time_step_ns=float(g["time_step_ns"]))
    bands = g["bands"]
    comp = SourceCompiler(g["wavelengths_nm"][bands], g["phase_index"], g["scale"][bands],
                          int(g["source_degree"]), int(g["azimuthal_degree"]), g["omega_per_ns"],
                          settings=settings)
    frame = ((g["frame_centre_m"], g["frame_axis"], g["frame_first"], g["frame_second"])
             if frame_from_fixture else None)
    return g, comp.compile(elements, frame)


def test_source_compile_matches_reference_node_sources():
    g, (points, channels, n_points, reference, frame) = compiled()
    n_points = n_points.cpu().numpy()
    for b in range(len(g["bands"])):
        ref_ch = g[f"band{b}_channels"]
        n = len(ref_ch)
        assert n_points[b] == n
        pts = points[b, :n].cpu().numpy()
        assert np.abs(pts[:, 0] - g[f"band{b}_z_m"]).max() < 1e-12
        assert np.abs(pts[:, 1:] - g[f"band{b}_transverse_m"]).max() < 1e-12
        ch = channels[b, :n].cpu().numpy()
        scale = np.abs(ref_ch).max()
        assert np.abs(ch - ref_ch).max() <= SOURCE_TOL * scale
        assert reference == pytest.approx(float(g[f"band{b}_reference_ns"]), abs=0)


def test_source_frame_restates_axis_frame():
    g, (_, _, _, _, frame) = compiled(frame_from_fixture=False)
    for got, key in zip(frame, ("frame_centre_m", "frame_axis", "frame_first", "frame_second")):
        assert np.abs(np.asarray(got) - g[key]).max() < 1e-12
