"""Write the flash fixtures from the reference's own float64 route.

Run here (reference present):  python tests/golden/make_flash_golden.py

Outputs
* ``lighthit_b200/tables/flash_450nm_2-250m.npz``: the multipole response table
  (``ResponseCache.moments``, radii, frequencies, medium band at 450 nm) that
  the reference builds with ``TransportKernel.build`` for the calibration-flash
  workload. It is the read-only input the device layout is built from.
* ``tests/golden/flash_c1.npz``: ``TransportKernel.transport(IsotropicFlash)``
  responses (reference ``transport.py:1061-1164``) for flashes drawn like the
  4096-flash workload (seed 11), plus two edge cases: a dim far flash with OMs
  outside the table's radial range, and the arguments of a flash that must
  raise (bright and out of range).
* ``tests/golden/readout_c0.npz``: ``readout_bins`` (``readout.py:43-72``) of
  seeded random relative spectra on the 65 -> 321 node grid and 160 bins.
"""
import json
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from _refenv import REPO, WORK, use_reference  # noqa: E402

sys.path.insert(0, str(REPO))
from lighthit_b200.workloads import flash_positions  # noqa: E402

lh = use_reference()
from lighthit.examples.synthetic import baikal_like_detector, synthetic_medium_model  # noqa: E402
from lighthit.readout import readout_bins  # noqa: E402

OMEGA = np.linspace(0.0, 1.2, 65)
READOUT = np.linspace(0.0, 1.2, 321)
EDGES = np.arange(-60.0, 745.0, 5.0)


def kernel(radial_high):
    medium = synthetic_medium_model()
    detector = baikal_like_detector(clusters=1)
    config = lh.KernelConfig(
        omega_per_ns=OMEGA, readout_omega_per_ns=READOUT, relative_time_edges_ns=EDGES,
        wavelength_nodes=3, scattering_degree=8, source_degree=8, azimuthal_degree=2,
        radial_range_m=(2.0, radial_high), radial_nodes=48, k_max_per_m=4.0,
        k_panel_per_m=0.1, k_order=6, threshold_pe=0.01,
        cache_directory=str(WORK / f"flash-cache-{radial_high:g}"), cache_policy="build")
    return lh.TransportKernel(medium, detector, config)


def main():
    k = kernel(250.0)
    detector = k.detector
    centre = lh.describe_geometry(detector).centroid_m
    positions = flash_positions(4096, centre, seed=11)
    k.build(source=lh.IsotropicFlash.monochromatic(positions[0], 1e10, 450.0))
    cache = k._cache_for(450.0)
    band = cache.medium
    tables = REPO / "lighthit_b200" / "tables"
    tables.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(
        tables / "flash_450nm_2-250m.npz",
        omega_per_ns=np.asarray(cache.grid.omega_per_ns, float),
        radii_m=np.asarray(cache.grid.radii_m, float),
        moments=np.asarray(cache.moments, np.complex128),
        absorption_per_m=band.absorption_per_m, scattering_per_m=band.scattering_per_m,
        g=band.g, group_index=band.group_index, wavelength_nm=band.wavelength_nm,
        radial_phase=str(cache.radial_phase), degree=int(cache.degree),
        provenance=json.dumps({
            "built_by": "lighthit TransportKernel.build (reference float64 route)",
            "medium": "lighthit.examples.synthetic.synthetic_medium_model",
            "kernel": {"scattering_degree": 8, "source_degree": 8, "azimuthal_degree": 2,
                       "radial_range_m": [2.0, 250.0], "radial_nodes": 48,
                       "k_max_per_m": 4.0, "k_panel_per_m": 0.1, "k_order": 6,
                       "wavelength_nm": 450.0}}))

    alpha = np.asarray(lh.cache.acceptance_coefficients(detector.angular_acceptance, cache.degree))
    picks = list(range(12))
    flashes = [(positions[i], 1e10, 0.0) for i in picks]
    # edge: a dim flash far outside the array (some OMs beyond 250 m, below the
    # absorption-only bound) and one at a nonzero emission time
    flashes.append((centre + np.array([0.0, 0.0, 330.0]), 1e6, 0.0))
    flashes.append((positions[12], 3e9, 17.5))
    spectra, comps, charges, origins, actives = [], [], [], [], []
    for pos, photons, t in flashes:
        r = k.transport(lh.IsotropicFlash.monochromatic(pos, photons, 450.0, time_ns=t))
        spectra.append(r.spectrum_pe.astype(np.complex128))
        comps.append(r.components_pe)
        charges.append(r.charge_components_pe)
        origins.append(r.time_origin_ns)
        actives.append(r.active)
    # edge: bright flash out of range must raise
    raise_pos = centre + np.array([0.0, 0.0, 330.0])
    try:
        k.transport(lh.IsotropicFlash.monochromatic(raise_pos, 1e10, 450.0))
        raised = ""
    except ValueError as exc:
        raised = str(exc)
    golden = REPO / "tests" / "golden"
    np.savez_compressed(
        golden / "flash_c1.npz",
        flash_position_m=np.array([f[0] for f in flashes]),
        flash_photons=np.array([f[1] for f in flashes]),
        flash_time_ns=np.array([f[2] for f in flashes]),
        spectrum_pe=np.array(spectra).astype(np.complex64),
        components_pe=np.array(comps).astype(np.float32),
        charge_components_pe=np.array(charges), time_origin_ns=np.array(origins),
        active=np.array(actives), alpha=alpha,
        om_positions_m=detector.positions_m, om_orientations=detector.orientations,
        om_area_m2=np.broadcast_to(np.asarray(detector.effective_area_m2, float),
                                   (len(detector),)).copy(),
        spectral_weight_450=float(detector.spectral_weight(450.0)),
        threshold_pe=0.01, edges_ns=EDGES, omega_per_ns=OMEGA, readout_omega_per_ns=READOUT,
        raise_position_m=raise_pos, raise_message=raised,
        first_positions_m=positions[:64])

    rng = np.random.default_rng(5)
    rel = (rng.normal(size=(65, 10)) + 1j * rng.normal(size=(65, 10))) * np.exp(
        -np.linspace(0, 4, 65))[:, None]
    rel[0] = rel[0].real
    bins = readout_bins(OMEGA, rel, EDGES, READOUT)
    np.savez_compressed(golden / "readout_c0.npz", relative=rel, bins=bins,
                        omega_per_ns=OMEGA, readout_omega_per_ns=READOUT, edges_ns=EDGES)
    print("flash fixtures:", len(flashes), "raise:", raised[:80])


if __name__ == "__main__":
    main()
