"""Write the order >=2 source-compile fixtures from the reference.

Run here (reference present):  python tests/golden/make_source_golden.py

Workload: the README-example shower (``make_shower_golden.setup`` settings,
without building the RTE tables). Calls the route's own
``node_sources`` (``shower/ge2.py:35-67`` -> ``compile_axial_slices``,
``_shower_basis.py:188-645``) with ``ShowerConfig().basis`` on the band fold
of rank 3 (``BandFold.of``) and the frame of the prompt steps
(``shower/api.py:373-402``).

Outputs ``tests/golden/source_c0.npz``: the fold's node bands, their
wavelengths, phase indices and scales; the frame and emission reference; the
compiled points and channels of every node band (all points at all 65
frequencies, complex64).
"""
import sys
from dataclasses import replace
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from _refenv import REPO, use_reference  # noqa: E402

lh = use_reference()
from lighthit.axial_source import AxisFrame  # noqa: E402
from lighthit.band_fold import BandFold  # noqa: E402
from lighthit.examples.synthetic import baikal_like_detector, synthetic_medium_model  # noqa: E402
from lighthit.shower.api import ShowerConfig  # noqa: E402
from lighthit.shower.ge2 import node_sources  # noqa: E402

OMEGA = np.linspace(0.0, 1.2, 65)


def main():
    medium = synthetic_medium_model()
    detector = baikal_like_detector(clusters=1)
    config = lh.KernelConfig(
        omega_per_ns=OMEGA, readout_omega_per_ns=np.linspace(0.0, 1.2, 321),
        relative_time_edges_ns=np.arange(-60.0, 745.0, 5.0), wavelength_nodes=3,
        scattering_degree=8, source_degree=8, azimuthal_degree=2, radial_range_m=(2.0, 150.0),
        radial_nodes=48, k_max_per_m=4.0, k_panel_per_m=0.1, k_order=6, threshold_pe=0.01)
    kernel = lh.TransportKernel(medium, detector, config)
    centre = lh.describe_geometry(detector).centroid_m
    pose = lh.SourcePose(centre + np.asarray([-12.0, 8.0, 0.0]), [0.35, -0.15, 0.925])
    shower = replace(lh.SyntheticShower.gaussian(pose, charged_track_length_m=300.0,
                                                 elements=2000, seed=7).elements,
                     cone_model="spectral")
    cfg = ShowerConfig()
    fold = BandFold.of(kernel, rank=int(cfg.band_rank))
    wavelengths = np.asarray(kernel.wavelength.wavelength_nm, float)
    sample = kernel.medium.sample(wavelengths)
    max_phase = float(np.max(sample["phase_index"]))
    elements = shower
    assert np.all(elements.beta * max_phase > 1)
    reference = elements.field(0, phase_index=max_phase)
    frame = AxisFrame.of(reference)
    sources = node_sources(kernel, elements, cfg.basis, fold, OMEGA, frame, reference)
    out = {}
    for b, s in enumerate(sources):
        out[f"band{b}_z_m"] = np.asarray(s.z_m, float)
        out[f"band{b}_transverse_m"] = np.asarray(s.transverse_m, float)
        out[f"band{b}_channels"] = np.asarray(s.channels, np.complex64)
        out[f"band{b}_reference_ns"] = float(s.reference_ns)
    np.savez_compressed(
        REPO / "tests" / "golden" / "source_c0.npz", bands=np.asarray(fold.bands, np.int64),
        scale=np.asarray(fold.scale, float), phase_index=np.asarray(fold.phase_index, float),
        wavelengths_nm=wavelengths, frame_centre_m=frame.centre_m, frame_axis=frame.axis,
        frame_first=frame.first, frame_second=frame.second, omega_per_ns=OMEGA,
        cell_m=cfg.basis.cell_m, axial_order=cfg.basis.axial_order, stencil_m=cfg.basis.stencil_m,
        stencil_threshold_m=cfg.basis.stencil_threshold_m, time_step_ns=cfg.basis.time_step_ns,
        source_degree=int(kernel.config.source_degree),
        azimuthal_degree=int(kernel.config.azimuthal_degree), **out)
    print("bands", fold.bands, "scale", fold.scale, "points", [len(s.z_m) for s in sources],
          "summary", sources[0].metadata if hasattr(sources[0], "metadata") else "")


if __name__ == "__main__":
    main()
