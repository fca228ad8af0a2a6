"""Write the two-shower event fixture from the reference's own float64 route.

Run here (reference present):  python tests/golden/make_event_golden.py

``EventTransport`` (``event.py:94-296``) on the README configuration (48-OM
array, 2-150 m tables): the README shower (2000 Gaussian elements, seed 7)
and a second copy of it moved SHIFT_M and delayed DELAY_NS, as two shower
components of one event: one clock, one OM selection, completion rounds on
receiver subsets.

Output ``tests/golden/event_c0.npz``: the recipe, the event response (charge,
bins float32, spectrum complex64, clocks, active) and the rounds.
"""
import json
import sys
from dataclasses import replace
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from make_shower_golden import setup  # noqa: E402  (builds the tables when missing)

from lighthit.event import EventTransport, SourceComponent  # noqa: E402
from lighthit.shower import ShowerData  # noqa: E402

SHIFT_M = np.array([6.0, -9.0, 14.0])
DELAY_NS = 35.0


def main():
    kernel, shower, cache = setup()
    second = replace(shower, start_m=np.asarray(shower.start_m) + SHIFT_M,
                     start_ns=np.asarray(shower.start_ns) + DELAY_NS,
                     end_ns=np.asarray(shower.end_ns) + DELAY_NS)
    event = EventTransport(kernel, shower_data=ShowerData.of(str(cache), str(cache / "ge2-pack")))
    r = event([SourceComponent("shower", shower, label="a"),
               SourceComponent("shower", second, label="b")])
    rounds = r.metadata["completion_rounds"]
    print(int(r.active.sum()), r.charge_components_pe.sum(axis=0), rounds)
    np.savez_compressed(
        Path(__file__).resolve().parent / "event_c0.npz", shift_m=SHIFT_M, delay_ns=DELAY_NS,
        charge_components_pe=r.charge_components_pe,
        components_pe=r.components_pe.astype(np.float32),
        spectrum_ge2_pe=r.spectrum_ge2_pe.astype(np.complex64),
        time_origin_ns=r.time_origin_ns, active=r.active, rounds=json.dumps(rounds))


if __name__ == "__main__":
    main()
