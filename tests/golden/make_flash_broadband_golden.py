"""Write the broadband-flash tables and fixtures from the reference's float64 route.

Run here (reference present):  python tests/golden/make_flash_broadband_golden.py

A broadband ``IsotropicFlash`` (``sources.py:81-107``) is transported at the
kernel's wavelength nodes: ``_flash_nodes`` (``transport.py:1049-1059``) gives
node photons ``photons * weight * shape / (weight . shape)``, every node adds
its own multipole spectrum, attenuation, flight time and order-0 arrival, and
the OM clock takes the fastest node (``transport.py:1088-1164``). The kernel
is the calibration-flash one of ``make_flash_golden.py`` (3 wavelength nodes,
2-250 m, 48 radial nodes).

Outputs
* ``lighthit_b200/tables/flash_<node>nm_2-250m.npz`` for the two nodes besides
  450 nm (the 450 nm table is ``make_flash_golden.py``'s), same fields;
* ``tests/golden/flash_broadband_c1.npz``: node wavelengths and weights, and
  the responses of eight flashes of the seed-11 workload (plus one at a
  nonzero time) with the spectral shape ``shape(lambda) = exp(-((lambda -
  SHAPE_CENTRE) / SHAPE_WIDTH)^2)``.
"""
import json
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from _refenv import REPO  # noqa: E402
from make_flash_golden import kernel, lh  # noqa: E402  (puts the reference on the path)

sys.path.insert(0, str(REPO))
from lighthit_b200.workloads import flash_positions  # noqa: E402

SHAPE_CENTRE, SHAPE_WIDTH = 440.0, 30.0


def shape(wavelength_nm):
    return np.exp(-((np.asarray(wavelength_nm, float) - SHAPE_CENTRE) / SHAPE_WIDTH) ** 2)


def export(cache, path):
    band = cache.medium
    np.savez_compressed(
        path, omega_per_ns=np.asarray(cache.grid.omega_per_ns, float),
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
                       "wavelength_nm": float(band.wavelength_nm)}}))


def main():
    k = kernel(250.0)
    centre = lh.describe_geometry(k.detector).centroid_m
    positions = flash_positions(4096, centre, seed=11)
    k.build(source=lh.IsotropicFlash.broadband(positions[0], 1e10, shape))
    nodes = np.asarray(k.wavelength.wavelength_nm, float)
    weights = np.asarray(k.wavelength.weight_nm, float)
    tables = REPO / "lighthit_b200" / "tables"
    for node in nodes:
        if abs(node - 450.0) > 1e-9:
            export(k._cache_for(float(node)), tables / f"flash_{node:.2f}nm_2-250m.npz")
    flashes = [(positions[i], 1e10, 0.0) for i in range(8)]
    flashes.append((positions[8], 4e9, 12.5))
    out = {k2: [] for k2 in ("spectrum", "components", "charge", "origin", "active")}
    for pos, photons, t in flashes:
        r = k.transport(lh.IsotropicFlash.broadband(pos, photons, shape, time_ns=t))
        out["spectrum"].append(r.spectrum_pe.astype(np.complex64))
        out["components"].append(r.components_pe.astype(np.float32))
        out["charge"].append(r.charge_components_pe)
        out["origin"].append(r.time_origin_ns)
        out["active"].append(r.active)
        print(int(r.active.sum()), r.charge_components_pe.sum(axis=0), r.metadata["wavelength_nm"])
    np.savez_compressed(
        REPO / "tests" / "golden" / "flash_broadband_c1.npz",
        node_wavelength_nm=nodes, node_weight_nm=weights,
        shape_centre_nm=SHAPE_CENTRE, shape_width_nm=SHAPE_WIDTH,
        flash_position_m=np.array([f[0] for f in flashes]),
        flash_photons=np.array([f[1] for f in flashes]),
        flash_time_ns=np.array([f[2] for f in flashes]),
        spectrum_pe=np.array(out["spectrum"]), components_pe=np.array(out["components"]),
        charge_components_pe=np.array(out["charge"]), time_origin_ns=np.array(out["origin"]),
        active=np.array(out["active"]))


if __name__ == "__main__":
    main()
