"""Write the delayed-light shower fixture from the reference's own float64 route.

Run here (reference present):  python tests/golden/make_shower_delayed_golden.py

Workload: the README shower of ``make_shower_golden.py`` (48-OM array, 2000
Gaussian elements, seed 7) plus delayed copies of some of its steps, the way
late neutron captures or decays follow a shower: elements DELAYED_A re-emitted
DELAY_A ns after their own time and elements BEYOND far beyond the readout
window. The reference route splits them with ``delay_groups``
(``shower/ge2.py:122-147``): delayed groups in the window (their own clocks and
shifted bin edges, ``shower/api.py:438-477``) and steps whose light cannot
arrive before the window ends (all-time charge only). Orders 0 and 1 take every
step; the copies share cells with the prompt steps, so their pencils mix times
and multiply the order-1 groups per OM (a second copy set at 135 ns took the
device route past its 8192 groups per OM).

Output ``tests/golden/shower_delayed_c0.npz``: the recipe (indices and delays),
the response's per-order charge, bins (float32), spectrum, clocks, active mask,
``ge2_charge_level`` and the delayed-light metadata.
"""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from make_shower_golden import setup  # noqa: E402  (builds the tables when missing)

import lighthit as lh  # noqa: E402
from lighthit.shower import ShowerData, ShowerTransport  # noqa: E402

DELAY_A, DELAY_BEYOND = 60.0, 5000.0
DELAYED_A = np.arange(500, 1100, 2)
BEYOND = np.arange(900, 960, 3)


def delayed_elements(base):
    """Base elements followed by the delayed copies (same geometry, later times)."""
    def field(name):
        return np.asarray(getattr(base, name))
    parts = [np.arange(len(field("beta"))), DELAYED_A, BEYOND]
    delays = [0.0, DELAY_A, DELAY_BEYOND]
    cat = {}
    for name in ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
                 "start_ns", "end_ns"):
        cat[name] = np.concatenate([field(name)[idx] + (d if name.endswith("_ns") else 0.0)
                                    for idx, d in zip(parts, delays)])
    n = len(cat["beta"])
    return lh.SpectralLightElements(
        cat["start_m"], cat["direction"], cat["length_m"], cat["coefficient0"],
        cat["coefficient2"], cat["beta"], cat["start_ns"], cat["end_ns"], np.arange(n),
        np.zeros(n, np.int64), 1.35, None, "spectral")


def main():
    kernel, shower, cache = setup()
    route = ShowerTransport(kernel, ShowerData.of(str(cache), str(cache / "ge2-pack")))
    elements = delayed_elements(shower)
    response = route(elements)
    meta = response.metadata["delayed_light"]
    print(meta, int(response.active.sum()), response.charge_components_pe.sum(axis=0))
    np.savez_compressed(
        Path(__file__).resolve().parent / "shower_delayed_c0.npz",
        delayed_a=DELAYED_A, beyond=BEYOND, delays=np.array([DELAY_A, DELAY_BEYOND]),
        charge_components_pe=response.charge_components_pe,
        components_pe=response.components_pe.astype(np.float32),
        spectrum_ge2_pe=response.spectrum_ge2_pe.astype(np.complex64),
        time_origin_ns=response.time_origin_ns, active=response.active,
        ge2_charge_level=np.asarray(response.metadata["ge2_charge_level"], np.int8),
        groups_in_window=int(meta["groups_in_window"]),
        steps_beyond_window=int(meta["steps_beyond_window"]),
        delayed_charge_pe=float(meta["delayed_charge_pe"]))


if __name__ == "__main__":
    main()
