"""Write the config-2 shower fixtures from the reference's own float64 route.

Run here (reference present), after ``python lighthit_b200/tables/build_tables.py c2``
has built the reference's 384-OM caches (2-450 m, 60 radial nodes, k panel 2 pi/450):

    python tests/golden/make_shower_c2_golden.py

Workload: the first 12 showers of the seeded config-2 stream
(``lighthit_b200.workloads.shower_stream`` and ``gaussian_shower``: element
counts log-uniform in 500-50000, 0.15 m of charged track per element, vertices
in a 200 m x 600 m cylinder around the array centroid, isotropic directions),
each through the reference ``ShowerTransport`` (``shower/api.py:222-288``) with
its default ``ShowerConfig``. The reference's wall time per shower (Numba, all
host threads, JIT warmed on a first shower that is not stored) is kept too.

Output ``tests/golden/shower_c2.npz`` per shower ``k``: ``s{k}_elements``,
``s{k}_checksum`` (sum of start_m and start_ns of the generated elements, to
catch generator drift), ``s{k}_charge`` (OM, 3), ``s{k}_active``,
``s{k}_origin`` (time_origin_ns), ``s{k}_active_ids`` and
``s{k}_components`` (active OMs, bins, 3) float32, ``s{k}_seconds``.
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

N_SHOWERS = 12
CACHE = _refenv_table_work() / "shower-c2"


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
        raise SystemExit(f"{CACHE} missing: run lighthit_b200/tables/build_tables.py c2 first")
    medium = synthetic_medium_model()
    detector = baikal_like_detector(clusters=8)
    config = lh.KernelConfig(
        omega_per_ns=np.linspace(0, 1.2, 65), readout_omega_per_ns=np.linspace(0, 1.2, 321),
        relative_time_edges_ns=np.arange(-60.0, 745.0, 5.0), wavelength_nodes=3,
        scattering_degree=8, source_degree=8, azimuthal_degree=2, radial_range_m=(2.0, 450.0),
        radial_nodes=60, k_max_per_m=4.0, k_panel_per_m=2 * np.pi / 450.0, k_order=6,
        threshold_pe=0.01, cache_directory=str(CACHE), cache_policy="require")
    kernel = lh.TransportKernel(medium, detector, config)
    route = ShowerTransport(kernel, ShowerData.of(str(CACHE), str(CACHE / "ge2-pack")))
    stream = shower_stream(N_SHOWERS, np.asarray(detector.positions_m).mean(axis=0))
    route(elements(stream[0])[1])  # JIT warm-up, not timed
    out = {}
    for k, s in enumerate(stream):
        el, src = elements(s)
        began = time.perf_counter()
        r = route(src)
        seconds = time.perf_counter() - began
        ids = np.flatnonzero(r.active)
        out.update({f"s{k}_elements": np.int64(s["elements"]),
                    f"s{k}_checksum": np.float64(el["start_m"].sum() + el["start_ns"].sum()),
                    f"s{k}_charge": np.asarray(r.charge_components_pe, float),
                    f"s{k}_active": np.asarray(r.active, bool),
                    f"s{k}_origin": np.asarray(r.time_origin_ns, float),
                    f"s{k}_active_ids": ids.astype(np.int32),
                    f"s{k}_components": np.asarray(r.components_pe, float)[ids].astype(np.float32),
                    f"s{k}_seconds": np.float64(seconds)})
        print(k, s["elements"], f"{seconds:.2f} s", len(ids), float(r.charge_pe.sum()), flush=True)
    out["threads"] = np.int64(os.cpu_count())
    np.savez_compressed(Path(__file__).resolve().parent / "shower_c2.npz", **out)


if __name__ == "__main__":
    main()
