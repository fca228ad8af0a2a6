"""Write the config-3 (high-resolution) shower fixtures from the reference's float64 route.

Run here (reference present), after ``python lighthit_b200/tables/build_tables.py c3``
has built the reference's 384-OM caches (1-300 m, 96 radial nodes, k panel 2 pi/300,
8 wavelength nodes, scattering/source degree 16, azimuthal degree 4, 1025 readout
nodes, 1 ns bins from -60 to 2000 ns):

    python tests/golden/make_shower_c3_golden.py

Workload: the first N_SHOWERS showers of the seeded config-3 stream
(``lighthit_b200.workloads.shower_stream`` with seed 31 and 20000 elements per
shower, 0.15 m of charged track per element, vertices in a 200 m x 600 m
cylinder around the array centroid, isotropic directions), each through the
reference ``ShowerTransport`` with its default ``ShowerConfig`` (band fold of
rank 3 over the 8 wavelength nodes). A shower the reference rejects (an OM
beyond the 300 m radial range with a conservative estimate above threshold,
``prompt.py:615-619``) is stored as ``s{k}_raises`` with the message.

Output ``tests/golden/shower_c3.npz`` per shower ``k``: ``s{k}_checksum``,
``s{k}_charge`` (OM, 3), ``s{k}_active``, ``s{k}_origin``, ``s{k}_active_ids``,
``s{k}_components`` (active OMs, bins, 3) float32, ``s{k}_spectrum`` (65,
active OMs) complex64, ``s{k}_level`` (ge2_charge_level), ``s{k}_seconds``.
"""
import os
import sys
import time
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from _refenv import REPO, table_work as _refenv_table_work, use_reference  # noqa: E402

lh = use_reference()
sys.path.insert(0, str(REPO))
from lighthit.examples.synthetic import baikal_like_detector, synthetic_medium_model  # noqa: E402
from lighthit.shower import ShowerData, ShowerTransport  # noqa: E402

from lighthit_b200.workloads import gaussian_shower, shower_stream  # noqa: E402

N_SHOWERS = int(os.environ.get("C3_SHOWERS", "4"))
CACHE = _refenv_table_work() / "shower-c3"


def elements(s):
    el = gaussian_shower(s["position_m"], s["direction"],
                         charged_track_length_m=s["charged_track_length_m"],
                         elements=s["elements"], seed=s["seed"])
    n = len(el["beta"])
    return el, lh.SpectralLightElements(
        el["start_m"], el["direction"], el["length_m"], el["coefficient0"], el["coefficient2"],
        el["beta"], el["start_ns"], el["end_ns"], np.arange(n), np.zeros(n, np.int64), 1.35,
        None, "spectral")


def main():
    if not CACHE.exists():
        raise SystemExit(f"{CACHE} missing: run lighthit_b200/tables/build_tables.py c3 first")
    medium = synthetic_medium_model()
    detector = baikal_like_detector(clusters=8)
    config = lh.KernelConfig(
        omega_per_ns=np.linspace(0, 1.2, 65), readout_omega_per_ns=np.linspace(0, 1.2, 1025),
        relative_time_edges_ns=np.arange(-60.0, 2000.5, 1.0), wavelength_nodes=8,
        scattering_degree=16, source_degree=16, azimuthal_degree=4, radial_range_m=(1.0, 300.0),
        radial_nodes=96, k_max_per_m=4.0, k_panel_per_m=2 * np.pi / 300.0, k_order=6,
        threshold_pe=0.01, cache_directory=str(CACHE), cache_policy="require")
    kernel = lh.TransportKernel(medium, detector, config)
    route = ShowerTransport(kernel, ShowerData.of(str(CACHE), str(CACHE / "ge2-pack")))
    stream = shower_stream(N_SHOWERS, np.asarray(detector.positions_m).mean(axis=0), seed=31,
                           low_elements=20000, high_elements=20000)
    out = {}
    for k, s in enumerate(stream):
        el, src = elements(s)
        out[f"s{k}_checksum"] = np.float64(el["start_m"].sum() + el["start_ns"].sum())
        began = time.perf_counter()
        try:
            r = route(src)
        except ValueError as error:
            out[f"s{k}_raises"] = np.array(str(error))
            print(k, "raises:", error, flush=True)
            continue
        seconds = time.perf_counter() - began
        ids = np.flatnonzero(r.active)
        out.update({f"s{k}_charge": np.asarray(r.charge_components_pe, float),
                    f"s{k}_active": np.asarray(r.active, bool),
                    f"s{k}_origin": np.asarray(r.time_origin_ns, float),
                    f"s{k}_active_ids": ids.astype(np.int32),
                    f"s{k}_components": np.asarray(r.components_pe, float)[ids].astype(np.float32),
                    f"s{k}_spectrum": np.asarray(r.spectrum_ge2_pe)[:, ids].astype(np.complex64),
                    f"s{k}_level": np.asarray(r.metadata["ge2_charge_level"], np.int8),
                    f"s{k}_seconds": np.float64(seconds)})
        print(k, f"{seconds:.2f} s", len(ids), float(r.charge_pe.sum()),
              r.charge_components_pe.sum(axis=0), "near" in str(r.metadata.get("near_field")),
              flush=True)
    out["threads"] = np.int64(os.cpu_count())
    out["n_showers"] = np.int64(N_SHOWERS)
    np.savez_compressed(Path(__file__).resolve().parent / "shower_c3.npz", **out)


if __name__ == "__main__":
    main()
