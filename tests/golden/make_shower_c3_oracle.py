"""Write the CPU oracle's response for the config-3 shower the reference rejects.

    python tests/golden/make_shower_c3_oracle.py

Shower 11 of the seeded config-3 stream makes the reference's control-variate
order 0 raise (its disk quadrature does not converge at order 64; recorded as
``s11_raises`` in ``shower_c3.npz``). The reference's direct ray form of order 0
(``_surface_ballistic_rays.evaluate``), which the oracle restates with the
reference's adaptive doubling, converges there; this script stores the oracle's
whole-route response of that shower (``oracle.shower.Route``, adaptive order 0,
orders 1 and >=2 as pinned to the reference) as ``shower_c3_oracle.npz``. Needs
no reference: only the committed tables and the oracle.
"""
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO))

from lighthit_b200.workloads import gaussian_shower, shower_stream  # noqa: E402
from oracle.shower import Route  # noqa: E402

TABLES = REPO / "lighthit_b200" / "tables"
SHOWERS = (11,)


def main():
    route = Route(np.load(TABLES / "route_c3.npz"), np.load(TABLES / "ge2_fold_384om_1-300m.npz"),
                  np.load(TABLES / "near_c3.npz"), order0_gauss=None, threads=8)
    stream = shower_stream(12, route.positions.mean(axis=0), seed=31, low_elements=20000,
                           high_elements=20000)
    out = {}
    for k in SHOWERS:
        s = stream[k]
        el = gaussian_shower(s["position_m"], s["direction"],
                             charged_track_length_m=s["charged_track_length_m"],
                             elements=s["elements"], seed=s["seed"])
        began = time.perf_counter()
        r = route(el)
        ids = np.flatnonzero(r["active"])
        out.update({f"s{k}_checksum": np.float64(el["start_m"].sum() + el["start_ns"].sum()),
                    f"s{k}_charge": r["charge_components_pe"], f"s{k}_active": r["active"],
                    f"s{k}_origin": r["time_origin_ns"], f"s{k}_active_ids": ids,
                    f"s{k}_components": r["components_pe"][ids].astype(np.float32),
                    f"s{k}_spectrum": r["spectrum_ge2_pe"][:, ids].astype(np.complex64),
                    f"s{k}_level": r["ge2_charge_level"]})
        print(k, "active", len(ids), "seconds", time.perf_counter() - began, flush=True)
    np.savez_compressed(REPO / "tests" / "golden" / "shower_c3_oracle.npz", **out)


if __name__ == "__main__":
    main()
