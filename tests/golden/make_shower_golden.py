"""Write the shower-route fixtures from the reference's own float64 route.

Run here (reference present):  python tests/golden/make_shower_golden.py

The workload is the reference README example (48-OM synthetic array, one
Gaussian synthetic shower of 2000 elements, seed 7, 300 m charged track,
spectral cones), with the kernel settings of that example.

Outputs
* ``lighthit_b200/tables/ge2_fold_48om_2-150m.npz``: the band-folded order >=2
  kernels (``ShowerTransport.tables()['folded']``, ``band_fold.py:155-208``)
  the reference builds once; the device layout is made from it.
* ``tests/golden/shower_c0.npz``:
  - the full ``ShowerTransport`` response (``shower/api.py:321-637``);
  - the node-band axial sources of the prompt steps (``shower/ge2.py:35-67``)
    at the zero frequency for every basis point, and at all 65 frequencies
    for every 8th point;
  - ``apply_folded`` (``shower/ge2.py:99-119``) of both against every OM
    inside the radial window.
"""
import json
import sys
from dataclasses import replace
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from _refenv import REPO, WORK, use_reference  # noqa: E402

lh = use_reference()
from lighthit.axial_source import AxisFrame  # noqa: E402
from lighthit.band_fold import zero_frequency  # noqa: E402
from lighthit.examples.synthetic import baikal_like_detector, synthetic_medium_model  # noqa: E402
from lighthit.shower import ShowerData, ShowerTransport  # noqa: E402
from lighthit.shower.ge2 import apply_folded, delay_groups, node_sources  # noqa: E402
from lighthit.shower.api import ShowerConfig  # noqa: E402

OMEGA = np.linspace(0.0, 1.2, 65)
READOUT = np.linspace(0.0, 1.2, 321)
EDGES = np.arange(-60.0, 745.0, 5.0)


def setup():
    """The README-example kernel (built tables in the work folder) and shower."""
    cache = WORK / "shower-c0"
    medium = synthetic_medium_model()
    detector = baikal_like_detector(clusters=1)
    config = lh.KernelConfig(
        omega_per_ns=OMEGA, readout_omega_per_ns=READOUT, relative_time_edges_ns=EDGES,
        wavelength_nodes=3, scattering_degree=8, source_degree=8, azimuthal_degree=2,
        radial_range_m=(2.0, 150.0), radial_nodes=48, k_max_per_m=4.0, k_panel_per_m=0.1,
        k_order=6, threshold_pe=0.01, cache_directory=str(cache), cache_policy="build")
    kernel = lh.TransportKernel(medium, detector, config)
    centre = lh.describe_geometry(detector).centroid_m
    pose = lh.SourcePose(centre + np.asarray([-12.0, 8.0, 0.0]), [0.35, -0.15, 0.925])
    shower = replace(lh.SyntheticShower.gaussian(pose, charged_track_length_m=300.0,
                                                 elements=2000, seed=7).elements,
                     cone_model="spectral")
    if not (cache / "ge2-pack" / "pack.json").exists():
        kernel.build(source=shower)
        kernel.ge2_kernel_store().save(str(cache / "ge2-pack"))
    return kernel, shower, cache


def main():
    kernel, shower, cache = setup()
    route = ShowerTransport(kernel, ShowerData.of(str(cache), str(cache / "ge2-pack")))
    response = route(shower)
    tables = route.tables()
    folded, fold = tables["folded"], tables["fold"]
    k = route.kernel

    # -- the route's own source compile for the prompt steps (shower/api.py:373-402)
    cfg = ShowerConfig()
    elements = k._source_elements(shower)
    wavelengths = np.asarray(k.wavelength.wavelength_nm, float)
    sample = k.medium.sample(wavelengths)
    max_phase = float(np.max(sample["phase_index"]))
    elements = elements.subset(elements.beta * max_phase > 1) if not np.all(
        elements.beta * max_phase > 1) else elements
    prompt_mask, late_groups, beyond = delay_groups(
        elements, prompt_delay_ns=cfg.prompt_delay_ns, cell_ns=cfg.delayed_cell_ns,
        window_end_ns=float(EDGES[-1]), group_index_max=float(np.max(sample["group_index"])))
    part = elements if np.all(prompt_mask) else elements.subset(prompt_mask)
    reference = part.field(0, phase_index=max_phase)
    frame = AxisFrame.of(reference)
    sources = node_sources(k, part, cfg.basis, fold, OMEGA, frame, reference)

    positions = np.asarray(k.detector.positions_m, float)
    looks = np.ascontiguousarray(-k.detector.orientations, float)
    area = np.broadcast_to(np.asarray(k.detector.effective_area_m2, float), (len(positions),)).copy()
    alpha = np.ascontiguousarray(k.acceptance()["alpha"], float)
    low, high = k.config.radial_range_m
    zero = zero_frequency(folded)
    zero_sources = [replace(s, channels=np.ascontiguousarray(s.channels[:, :, :1])) for s in sources]
    spec_zero = apply_folded(zero, zero_sources, positions, looks, alpha, area, (low, high))
    keep = np.arange(0, len(sources[0].z_m), 8)
    sub = [replace(s, z_m=s.z_m[keep], transverse_m=s.transverse_m[keep],
                   channels=np.ascontiguousarray(s.channels[keep])) for s in sources]
    spec_sub = apply_folded(folded, sub, positions, looks, alpha, area, (low, high))

    tables_dir = REPO / "lighthit_b200" / "tables"
    np.savez_compressed(
        tables_dir / "ge2_fold_48om_2-150m.npz",
        coefficients=np.asarray(folded["coefficients"], np.complex64),
        log_r=np.asarray(folded["log_r"], float), omega=np.asarray(folded["omega"], float),
        absorption=np.asarray(folded["absorption"], float), speed=np.asarray(folded["speed"], float),
        degree=int(folded["degree"]), acceptance_degree=int(folded["acceptance_degree"]),
        pair_lambda=np.asarray(folded["pair_lambda"], np.int64),
        pair_mu=np.asarray(folded["pair_mu"], np.int64), phase=str(folded["phase"]),
        bands=np.asarray(fold.bands, np.int64), scale=np.asarray(fold.scale, float),
        provenance=json.dumps({"built_by": "lighthit ShowerTransport.tables() (BandFold rank 3)",
                               "kernel": {"radial_range_m": [2.0, 150.0], "radial_nodes": 48,
                                          "scattering_degree": 8, "source_degree": 8,
                                          "azimuthal_degree": 2, "wavelength_nodes": 3}}))

    def source_arrays(items, tag):
        out = {}
        out[f"{tag}_z_m"] = np.asarray(items[0].z_m, float)
        out[f"{tag}_transverse_m"] = np.asarray(items[0].transverse_m, float)
        out[f"{tag}_channels"] = np.stack([np.asarray(s.channels, np.complex64) for s in items])
        out[f"{tag}_reference_ns"] = np.array([float(s.reference_ns) for s in items])
        return out

    golden = REPO / "tests" / "golden"
    np.savez_compressed(
        golden / "shower_c0.npz",
        charge_components_pe=response.charge_components_pe,
        components_pe=response.components_pe.astype(np.float32),
        spectrum_ge2_pe=response.spectrum_ge2_pe.astype(np.complex64),
        time_origin_ns=response.time_origin_ns, active=response.active,
        ge2_charge_level=np.asarray(response.metadata["ge2_charge_level"], np.int8),
        frame_centre_m=frame.centre_m, frame_axis=frame.axis, frame_first=frame.first,
        frame_second=frame.second, om_positions_m=positions, om_looks=looks, om_area_m2=area,
        alpha=alpha, radial_window_m=np.array([low, high]),
        channel_degree=np.asarray(sources[0].channel_degree, np.int64),
        source_degree=int(sources[0].degree), azimuthal_degree=int(sources[0].azimuthal_degree),
        spec_zero=spec_zero.astype(np.complex128), spec_sub=spec_sub.astype(np.complex128),
        **source_arrays(zero_sources, "zero"), **source_arrays(sub, "sub"),
        n_points=len(sources[0].z_m), edges_ns=EDGES, omega_per_ns=OMEGA,
        readout_omega_per_ns=READOUT, threshold_pe=0.01)
    print("active", int(response.active.sum()), "charge", response.charge_components_pe.sum(axis=0),
          "points", len(sources[0].z_m), "sub", len(keep))


if __name__ == "__main__":
    main()
