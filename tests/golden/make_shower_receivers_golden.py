"""Write the receiver-subset fixture from the reference's own float64 route.

Run here (reference present):  python tests/golden/make_shower_receivers_golden.py

``ShowerTransport(...)(source, receivers=...)`` restricts the route to those
OMs with threshold zero (``shower/api.py:205-212``, ``subset_kernel``): every
receiver computed in full, the response covering only them. ``EventTransport``
uses it to refine OMs that the sum of an event's sources makes active, with
the event clock (``time_origin_ns``) and the other sources' light
(``selection_extra_charge``). Workload: the README shower (48-OM array, 2000
Gaussian elements, seed 7) on RECEIVERS, once with the full response's clocks
and EXTRA charges (``event``) and once with the route's own subset clock
(``plain``).

Output ``tests/golden/shower_receivers_c0.npz``.
"""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from make_shower_golden import setup  # noqa: E402  (builds the tables when missing)

from lighthit.shower import ShowerData, ShowerTransport  # noqa: E402

RECEIVERS = np.array([3, 7, 20, 21, 33, 40, 47])
EXTRA = np.array([0.0, 0.5, 0.0, 1.0, 0.0, 0.2, 0.0])


def main():
    kernel, shower, cache = setup()
    route = ShowerTransport(kernel, ShowerData.of(str(cache), str(cache / "ge2-pack")))
    full = route(shower)
    clock = full.time_origin_ns[RECEIVERS] - 3.0
    out = dict(receivers=RECEIVERS, extra=EXTRA, clock=clock)
    for name, kw in (("event", dict(time_origin_ns=clock, selection_extra_charge=EXTRA)),
                     ("plain", {})):
        r = route(shower, receivers=RECEIVERS, **kw)
        print(name, r.active.astype(int), r.charge_components_pe.sum(axis=0))
        out.update({f"{name}_charge": r.charge_components_pe,
                    f"{name}_components": r.components_pe.astype(np.float32),
                    f"{name}_spectrum": r.spectrum_ge2_pe.astype(np.complex64),
                    f"{name}_origin": r.time_origin_ns, f"{name}_active": r.active,
                    f"{name}_level": np.asarray(r.metadata["ge2_charge_level"], np.int8)})
    np.savez_compressed(Path(__file__).resolve().parent / "shower_receivers_c0.npz", **out)


if __name__ == "__main__":
    main()
