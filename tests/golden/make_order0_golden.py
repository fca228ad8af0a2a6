"""Write the order-0 (direct light) fixtures from the reference.

Run here (reference present):  python tests/golden/make_order0_golden.py
(after make_shower_golden.py, whose response fixture supplies the route's clock).

Workload: the README-example shower (48-OM synthetic array, 2000 Gaussian
elements, seed 7, spectral cones) of ``make_shower_golden.setup``.

Outputs ``tests/golden/order0_c0.npz``:
* the element arrays the prompt route integrates (``prompt.py:542-562``:
  ``_source_elements`` and the spectral-threshold subset);
* the optical panels of ``prepare_optics(..., exact_response=True)``
  (``ballistic_interval.py:64-161``), as ``PreparedBallistic`` builds them
  (``_surface_ballistic.py:36-37``);
* the detector arrays (positions, looks = -orientations, effective areas,
  sphere radii, acceptance Legendre coefficients);
* ``interval_candidates`` (``_ballistic_interval_numba.py:450-519``) with the
  sphere always in reach and the surface axis included, as
  ``PreparedBallistic`` calls it (``_surface_ballistic.py:38-40``);
* the reference's direct first-entry ray quadrature
  ``_surface_ballistic_rays.evaluate`` over those pairs at Gauss orders 8 and
  16, with the route's per-OM clock and the 5 ns edges;
* for every OM, the route's own order-0 charge and (active OMs) bins are in
  ``shower_c0.npz``.
"""
import sys
import time
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from make_shower_golden import EDGES, setup  # noqa: E402
from _refenv import REPO  # noqa: E402

from lighthit._ballistic_interval_numba import interval_candidates  # noqa: E402
from lighthit._surface_ballistic_rays import evaluate  # noqa: E402
from lighthit.ballistic_interval import BallisticIntervalConfig, prepare_optics  # noqa: E402


def main():
    kernel, shower, _ = setup()
    golden = REPO / "tests" / "golden"
    route = np.load(golden / "shower_c0.npz")
    elements = kernel._source_elements(shower)
    # prompt.py:542-562: drop steps below threshold at the critical wavelengths
    low, high = kernel.config.wavelength_range_nm or kernel.medium.wavelength_range_nm
    native = kernel.medium.wavelength_nm
    critical = np.r_[low, native[(native > low) & (native < high)], high]
    threshold_phase = float(np.max(kernel.medium.sample(critical)["phase_index"]))
    valid = elements.beta * threshold_phase > 1
    if not np.all(valid):
        elements = elements.subset(valid)
    tables = prepare_optics(kernel, BallisticIntervalConfig(), exact_response=True)
    d = kernel.detector
    n = len(d)
    positions = np.ascontiguousarray(d.positions_m, float)
    looks = np.ascontiguousarray(-d.orientations, float)
    areas = np.broadcast_to(np.asarray(d.effective_area_m2, float), (n,)).copy()
    radii = np.broadcast_to(np.asarray(d.receiver_surface.radii(n), float), (n,)).copy()
    alpha = np.ascontiguousarray(kernel.acceptance()["alpha"], float)
    arrays = {name: np.ascontiguousarray(getattr(elements, name), float) for name in
              ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
               "start_ns", "end_ns")}
    po, pe = interval_candidates(positions, radii, np.inf, arrays["start_m"],
                                 arrays["direction"], arrays["length_m"],
                                 arrays["coefficient0"], arrays["beta"],
                                 tables["phase_nodes"], True)
    origins = np.asarray(route["time_origin_ns"], float)
    out = {}
    for order in (8, 16):
        gx, gw = np.polynomial.legendre.leggauss(order)
        t0 = time.perf_counter()
        q, b = evaluate(po, pe, positions, looks, areas, radii, arrays["start_m"],
                        arrays["direction"], arrays["length_m"], arrays["coefficient0"],
                        arrays["coefficient2"], arrays["beta"], arrays["start_ns"],
                        arrays["end_ns"], tables["panel_edges"], tables["phase_nodes"],
                        tables["group_nodes"], tables["extinction_nodes"],
                        tables["efficiency_coefficients"], alpha, gx, gw, origins, EDGES)
        out[f"rays{order}_charge"] = q
        out[f"rays{order}_bins"] = b
        print(f"order {order}: {time.perf_counter() - t0:.1f} s, total {q.sum():.8f} pe")
    # a small pair subset at order 8, for tight checks of restatements
    sub = np.arange(0, len(po), 37)
    gx, gw = np.polynomial.legendre.leggauss(8)
    qs, bs = evaluate(po[sub], pe[sub], positions, looks, areas, radii, arrays["start_m"],
                      arrays["direction"], arrays["length_m"], arrays["coefficient0"],
                      arrays["coefficient2"], arrays["beta"], arrays["start_ns"],
                      arrays["end_ns"], tables["panel_edges"], tables["phase_nodes"],
                      tables["group_nodes"], tables["extinction_nodes"],
                      tables["efficiency_coefficients"], alpha, gx, gw, origins, EDGES)
    np.savez_compressed(
        golden / "order0_c0.npz", **arrays, positions_m=positions, looks=looks, areas_m2=areas,
        radii_m=radii, alpha=alpha, origins_ns=origins, edges_ns=EDGES,
        panel_edges=tables["panel_edges"], phase_nodes=tables["phase_nodes"],
        group_nodes=tables["group_nodes"], extinction_nodes=tables["extinction_nodes"],
        efficiency_coefficients=tables["efficiency_coefficients"], pair_om=po, pair_element=pe,
        sub_pairs=sub, sub8_charge=qs, sub8_bins=bs, **out)
    print("pairs", len(po), "elements", len(elements))


if __name__ == "__main__":
    main()
