"""Write the near-threshold shower fixture from the reference's own float64 route.

Run here (reference present):  python tests/golden/make_shower_threshold_golden.py

Workload: the README shower (48-OM array, 2000 Gaussian elements, seed 7) with
the speed of some of its elements lowered near the Cherenkov threshold, the
way the slow electrons of a real shower sit there: every element with index
= 0 mod 5 at BETA_BLUE (above threshold in the bluest of the three wavelength
nodes only: beta n = 1.0011, 0.9982, 0.9965) and every element = 1 mod 5 at
BETA_TWO (bluest and middle nodes: 1.0031, 1.0002, 0.9985), each with its own
coefficient2 = -coefficient0 / beta^2 and end time start + length / (beta c).
The reference evaluates order 1 as a fused unit of the elements emitting in
every band plus one unit per band for the rest (``prompt.py:683-719``,
``muon/secondary_first.py:184-204``), and compiles each node band's order >=2
source from its own emitting elements (``shower/ge2.py:21-67``).

Output ``tests/golden/shower_threshold_c0.npz``: the recipe and the response
(per-order charge, bins float32, spectrum complex64, clocks, active mask,
ge2_charge_level, order-1 level).
"""
import sys
from dataclasses import replace
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from make_shower_golden import setup  # noqa: E402  (builds the tables when missing)

from lighthit.shower import ShowerData, ShowerTransport  # noqa: E402

C_M_PER_NS = 0.299792458
BETA_BLUE, BETA_TWO = 0.7455, 0.7470


def slowed(shower):
    """The README shower with every fifth element (and the next) near threshold."""
    index = np.arange(len(shower.beta))
    beta = np.asarray(shower.beta, float).copy()
    beta[index % 5 == 0] = BETA_BLUE
    beta[index % 5 == 1] = BETA_TWO
    c0 = np.asarray(shower.coefficient0, float)
    length = np.asarray(shower.length_m, float)
    start_ns = np.asarray(shower.start_ns, float)
    return replace(shower, beta=beta, coefficient2=-c0 / beta ** 2,
                   end_ns=start_ns + length / (beta * C_M_PER_NS))


def main():
    kernel, shower, cache = setup()
    route = ShowerTransport(kernel, ShowerData.of(str(cache), str(cache / "ge2-pack")))
    moved = slowed(shower)
    response = route(moved)
    print(int(response.active.sum()), response.charge_components_pe.sum(axis=0),
          response.metadata.get("prompt_order1_level") is not None)
    np.savez_compressed(
        Path(__file__).resolve().parent / "shower_threshold_c0.npz",
        beta_blue=BETA_BLUE, beta_two=BETA_TWO,
        charge_components_pe=response.charge_components_pe,
        components_pe=response.components_pe.astype(np.float32),
        spectrum_ge2_pe=response.spectrum_ge2_pe.astype(np.complex64),
        time_origin_ns=response.time_origin_ns, active=response.active,
        ge2_charge_level=np.asarray(response.metadata["ge2_charge_level"], np.int8),
        prompt_order1_level=np.asarray(response.metadata["prompt_order1_level"], np.int8))


if __name__ == "__main__":
    main()
