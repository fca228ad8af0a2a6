"""Build the read-only tables of the shower route with the reference (run once, here).

    python lighthit_b200/tables/build_tables.py c0     # 48 OMs, 2-150 m, 48 radial nodes
    python lighthit_b200/tables/build_tables.py c2     # 384 OMs, 2-450 m, 60 radial nodes
    python lighthit_b200/tables/build_tables.py c2 near   # only near_c2.npz
    python lighthit_b200/tables/build_tables.py c3     # 384 OMs, 1-300 m, 8 wavelengths, L=16

The reference (LightHit, pure Python + Numba) builds its RTE caches
(``TransportKernel.build``) and the order >=2 kernel pack
(``ge2_kernel_store().save``); ``ShowerTransport.tables()`` folds them onto the
rank-3 node bands (``band_fold.py:155-208``). This script stores, for the
device route:
* ``ge2_fold_<n>om_<lo>-<hi>m.npz``: the folded order >=2 kernels;
* ``near_<config>.npz``: the first radial interval of the per-wavelength order
  >=2 kernels (``Ge2KernelStore.bundle``, not folded), the only part the
  near-field clamp reads (``near_field.py:91-171``: every point closer than the
  radial minimum takes the amplitude at that minimum);
* ``route_<config>.npz``: the kernel's medium and detector constants the route
  reads (wavelength nodes and weights, phase/group indices, absorption and
  scattering, detector spectral weights, the spectral-cut phase index of
  ``prompt.py:542-550``, the node bands' wavelengths, phases and fold scales,
  the prompt tables of ``prompt.py:412-434``, the first-entry optical panels of
  ``prepare_optics(..., exact_response=True)``, the acceptance coefficients,
  OM geometry and the kernel configuration).
It needs the reference sources (``LIGHTHIT_REFERENCE_SRC``) and a writable
Numba cache; the device route reads only the files it writes.
"""
import json
import os
import sys
from dataclasses import replace
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def _required(name, what):
    value = os.environ.get(name)
    if not value:
        raise SystemExit(f"set {name} to {what}")
    return Path(value)


BASE = dict(wavelength_nodes=3, degree=8, azimuthal_degree=2, readout_nodes=321,
            bin_ns=5.0, window_end_ns=740.0)
CONFIGS = {
    "c0": dict(BASE, clusters=1, radial_range_m=(2.0, 150.0), radial_nodes=48,
               k_panel_per_m=0.1),
    "c2": dict(BASE, clusters=8, radial_range_m=(2.0, 450.0), radial_nodes=60,
               k_panel_per_m=2 * np.pi / 450.0),
    # high-resolution precision study: 8 wavelength nodes, degree 16, azimuthal
    # degree 4, 96 radial nodes over 1-300 m, 1025 readout nodes, 1 ns bins to 2000 ns
    "c3": dict(clusters=8, radial_range_m=(1.0, 300.0), radial_nodes=96,
               k_panel_per_m=2 * np.pi / 300.0, wavelength_nodes=8, degree=16,
               azimuthal_degree=4, readout_nodes=1025, bin_ns=1.0, window_end_ns=2000.0),
}


def near_interval(route, tables):
    """The near-field table (a dict): interval 0 of every wavelength's order >=2
    spline of a reference ``ShowerTransport`` (``Ge2KernelStore.bundle``)."""
    from lighthit.shower_basis import _frequency_indices
    indices = _frequency_indices(route.kernel, route.config.frequency_nodes)
    bundle = tables["store"].bundle(route.kernel, indices)
    if bundle.get("phase") != "flight":
        raise ValueError("near-field table needs flight-phase splines")
    return dict(
        coefficients=np.ascontiguousarray(np.asarray(bundle["coefficients"])[:, 0], np.complex64),
        log_r=np.asarray(bundle["log_r"], float)[:2],
        radial_high_m=float(np.exp(np.asarray(bundle["log_r"], float)[-1])),
        omega=np.asarray(bundle["omega"], float),
        absorption=np.asarray(bundle["absorption"], float),
        speed=np.asarray(bundle["speed"], float), degree=int(bundle["degree"]),
        acceptance_degree=int(bundle["acceptance_degree"]),
        pair_lambda=np.asarray(bundle["pair_lambda"], np.int64),
        pair_mu=np.asarray(bundle["pair_mu"], np.int64),
        provenance=json.dumps({"built_by": "lighthit Ge2KernelStore.bundle (interval 0)",
                               "frequency_indices": np.asarray(indices).tolist()}))


def folded_kernels(route, tables):
    """The folded order >=2 kernels (a dict) of a reference ``ShowerTransport``
    (``ShowerTransport.tables()``, ``band_fold.py:155-208``)."""
    folded, fold = tables["folded"], tables["fold"]
    cfg = route.kernel.config
    lo, hi = (float(v) for v in cfg.radial_range_m)
    return dict(
        coefficients=np.asarray(folded["coefficients"], np.complex64),
        log_r=np.asarray(folded["log_r"], float), omega=np.asarray(folded["omega"], float),
        absorption=np.asarray(folded["absorption"], float), speed=np.asarray(folded["speed"], float),
        degree=int(folded["degree"]), acceptance_degree=int(folded["acceptance_degree"]),
        pair_lambda=np.asarray(folded["pair_lambda"], np.int64),
        pair_mu=np.asarray(folded["pair_mu"], np.int64), phase=str(folded["phase"]),
        bands=np.asarray(fold.bands, np.int64), scale=np.asarray(fold.scale, float),
        provenance=json.dumps({"built_by": "lighthit ShowerTransport.tables() (BandFold rank "
                                           f"{len(fold.bands)})",
                               "kernel": {"radial_range_m": [lo, hi],
                                          "radial_nodes": int(cfg.radial_nodes),
                                          "k_panel_per_m": float(cfg.k_panel_per_m)}}))


def route_constants(route, tables):
    """The route's medium and detector constants (a dict) of a reference
    ``ShowerTransport``: wavelength nodes and weights, phase/group indices,
    absorption and scattering, detector spectral weights, the spectral-cut phase
    index (``prompt.py:542-550``), the node bands, the prompt tables
    (``prompt.py:412-434``), the first-entry optical panels of
    ``prepare_optics(..., exact_response=True)``, the acceptance, OM geometry
    and the kernel configuration."""
    from lighthit.ballistic_interval import BallisticIntervalConfig, prepare_optics
    from lighthit.prompt import _spectral_tables
    k = route.kernel
    fold = tables["fold"]
    wl = np.asarray(k.wavelength.wavelength_nm, float)
    sample = k.medium.sample(wl)
    low, high = k.config.wavelength_range_nm or k.medium.wavelength_range_nm
    native = k.medium.wavelength_nm
    critical = np.r_[low, native[(native > low) & (native < high)], high]
    prompt = _spectral_tables(k)
    optics = prepare_optics(k, BallisticIntervalConfig(), exact_response=True)
    d = k.detector
    n_om = len(d)
    return dict(
        wavelength_nm=wl, weight_nm=np.asarray(k.wavelength.weight_nm, float),
        phase_index=np.asarray(sample["phase_index"], float),
        group_index=np.asarray(sample["group_index"], float),
        absorption_per_m=np.asarray(sample["absorption_per_m"], float),
        scattering_per_m=np.asarray(sample["scattering_per_m"], float),
        efficiency=np.asarray(d.spectral_weight(wl), float),
        threshold_phase=float(np.max(k.medium.sample(critical)["phase_index"])),
        g=float(k.medium.g), fold_bands=np.asarray(fold.bands, np.int64),
        fold_scale=np.asarray(fold.scale, float), fold_phase=np.asarray(fold.phase_index, float),
        mus=prompt["mus"], mut=prompt["mut"], speed=prompt["speed"], s0w=prompt["s0w"],
        s2w=prompt["s2w"], **{f"optics_{key}": optics[key] for key in (
            "panel_edges", "phase_nodes", "group_nodes", "extinction_nodes",
            "efficiency_coefficients")},
        alpha=np.asarray(k.acceptance()["alpha"], float),
        peak_acceptance=float(np.max(np.abs(np.asarray(
            d.angular_acceptance(np.linspace(-1, 1, 257)), float)))),
        positions_m=np.asarray(d.positions_m, float),
        looks=np.asarray(-d.orientations, float),
        areas_m2=np.broadcast_to(np.asarray(d.effective_area_m2, float), (n_om,)).copy(),
        radii_m=np.broadcast_to(np.asarray(d.receiver_surface.radii(n_om), float), (n_om,)).copy(),
        omega_per_ns=np.asarray(k.config.omega_per_ns, float),
        readout_omega_per_ns=np.asarray(k.config.readout_omega_per_ns, float),
        edges_ns=np.asarray(k.config.relative_time_edges_ns, float),
        radial_range_m=np.asarray(k.config.radial_range_m, float),
        threshold_pe=float(k.config.threshold_pe), source_degree=int(k.config.source_degree),
        azimuthal_degree=int(k.config.azimuthal_degree))


def main(name, near_only=False):
    src = _required("LIGHTHIT_REFERENCE_SRC", "the reference's src folder")
    work = _required("LIGHTHIT_TABLE_WORK", "a writable folder for the reference's RTE caches")
    os.environ.setdefault("NUMBA_CACHE_DIR", str(work / "numba-cache"))
    sys.path.insert(0, str(src))
    import lighthit as lh
    from lighthit.examples.synthetic import baikal_like_detector, synthetic_medium_model
    from lighthit.shower import ShowerData, ShowerTransport

    c = CONFIGS[name]
    cache = work / f"shower-{name}"
    medium = synthetic_medium_model()
    detector = baikal_like_detector(clusters=c["clusters"])
    omega = np.linspace(0.0, 1.2, 65)
    config = lh.KernelConfig(
        omega_per_ns=omega, readout_omega_per_ns=np.linspace(0.0, 1.2, c["readout_nodes"]),
        relative_time_edges_ns=np.arange(-60.0, c["window_end_ns"] + 0.5 * c["bin_ns"],
                                         c["bin_ns"]),
        wavelength_nodes=c["wavelength_nodes"], scattering_degree=c["degree"],
        source_degree=c["degree"], azimuthal_degree=c["azimuthal_degree"],
        radial_range_m=c["radial_range_m"], radial_nodes=c["radial_nodes"], k_max_per_m=4.0,
        k_panel_per_m=float(c["k_panel_per_m"]), k_order=6, threshold_pe=0.01,
        cache_directory=str(cache), cache_policy="build")
    kernel = lh.TransportKernel(medium, detector, config)
    centre = lh.describe_geometry(detector).centroid_m
    pose = lh.SourcePose(centre + np.asarray([-12.0, 8.0, 0.0]), [0.35, -0.15, 0.925])
    shower = replace(lh.SyntheticShower.gaussian(pose, charged_track_length_m=300.0,
                                                 elements=2000, seed=7).elements,
                     cone_model="spectral")
    if not (cache / "ge2-pack" / "pack.json").exists():
        kernel.build(source=shower)
        kernel.ge2_kernel_store().save(str(cache / "ge2-pack"))
    route = ShowerTransport(kernel, ShowerData.of(str(cache), str(cache / "ge2-pack")))
    tables = route.tables()
    np.savez_compressed(HERE / f"near_{name}.npz", **near_interval(route, tables))
    print("wrote", f"near_{name}.npz")
    if near_only:
        return
    lo, hi = c["radial_range_m"]
    np.savez_compressed(HERE / f"ge2_fold_{len(detector)}om_{lo:g}-{hi:g}m.npz",
                        **folded_kernels(route, tables))
    np.savez_compressed(HERE / f"route_{name}.npz", **route_constants(route, tables))
    print("wrote", name, "fold", tables["fold"].bands, tables["fold"].scale)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "c0",
         near_only=len(sys.argv) > 2 and sys.argv[2] == "near")
