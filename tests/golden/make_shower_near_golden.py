"""Write the near-field fixtures from the reference's own float64 code.

Run here (reference present):  python tests/golden/make_shower_near_golden.py

Two workloads on the README configuration (48-OM array, 2-150 m tables):

* ``pass``: the README shower (2000 Gaussian elements, seed 7) translated so
  that its closest element midpoint lies GAP_M from OM 20, well inside the 2 m
  radial minimum of the order >=2 tables. The reference's ``ShowerTransport``
  leaves the near basis points out of its table sums and adds them back with
  ``add_near_field`` (``shower/api.py:536-538``, ``near_field.py:174-217``).
  Stored: the full response and the near field alone (``near_field_ge2`` on the
  response clock).
* ``edges``: ``near_field_ge2`` alone (``near_field.py:91-171``) on hand-made
  elements around OM 20 and OM 21: a line through the OM centre (the
  transverse-axis branch), a 3 m element crossing the sphere (many panels),
  elements that start or end inside it, one above the Cherenkov threshold in
  the bluest band only, one with coefficient0 = 0, one whose coefficient2 makes
  the yield negative and one below threshold everywhere (portions without
  harmonics), one far away.

Output ``tests/golden/shower_near_c0.npz``.
"""
import sys
from dataclasses import replace
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from make_shower_golden import setup  # noqa: E402  (builds the tables when missing)

import lighthit as lh  # noqa: E402
from lighthit.near_field import near_field_ge2  # noqa: E402
from lighthit.shower import ShowerData, ShowerTransport  # noqa: E402
from lighthit.shower_basis import _frequency_indices  # noqa: E402

OM = 20
GAP_M = 1.0


def moved_shower(shower, positions):
    """The README shower translated so its closest element midpoint is GAP_M from OM."""
    start = np.asarray(shower.start_m, float)
    middle = start + 0.5 * np.asarray(shower.length_m)[:, None] * np.asarray(shower.direction)
    k = int(np.argmin(np.linalg.norm(middle - positions[OM], axis=1)))
    v = positions[OM] - middle[k]
    shift = v * (1.0 - GAP_M / np.linalg.norm(v))
    return replace(shower, start_m=start + shift), shift


def edge_elements(positions):
    """Hand-made elements around OM 20 and OM 21 (see the module docstring)."""
    p, q = positions[OM], positions[OM + 1]
    rows = []  # start, direction, length, c0, c2, beta, t0, t1

    def add(start, direction, length, c0=1.0e3, c2=-5.0e2, beta=1.0, t0=10.0):
        d = np.asarray(direction, float)
        d = d / np.linalg.norm(d)
        rows.append((np.asarray(start, float), d, float(length), c0, c2, beta, t0,
                     t0 + length / (beta * 0.299792458)))

    axis = np.array([0.2, -0.3, 0.93])
    add(p - 1.6 * axis / np.linalg.norm(axis), axis, 1.0)            # line through the centre
    add(p + [1.2, -1.5, -0.4], [0.1, 0.9, 0.2], 3.0, t0=25.0)         # crosses the sphere
    add(p + [0.3, 0.2, -0.5], [0.0, 0.6, 0.8], 2.5, t0=40.0)          # starts inside
    add(p + [-0.4, 1.9, 0.1], [0.3, -0.95, 0.0], 1.6, t0=5.0)         # ends inside
    add(p + [0.6, -0.6, 1.0], [0.7, 0.7, 0.1], 0.8, beta=0.7455)      # above threshold in the bluest band only
    add(p + [-0.8, 0.0, -1.2], [0.0, 0.0, 1.0], 1.0, c0=0.0, c2=-800.0)
    add(p + [0.9, -0.3, 0.2], [0.0, 1.0, 0.2], 0.7, c2=-3.0e3)     # negative yield
    add(p + [0.5, 0.5, 0.5], [1.0, 0.0, 0.0], 0.5, beta=0.5)          # no harmonics at all
    add(q + [0.9, 0.1, -1.1], [-0.2, 0.1, 0.97], 2.0, t0=60.0)        # the neighbouring OM
    add(p + [40.0, 0.0, 0.0], [0.0, 1.0, 0.0], 1.0)                   # far from every OM
    cols = list(zip(*rows))
    n = len(rows)
    return lh.SpectralLightElements(
        np.stack(cols[0]), np.stack(cols[1]), np.array(cols[2]), np.array(cols[3]),
        np.array(cols[4]), np.array(cols[5]), np.array(cols[6]), np.array(cols[7]),
        np.arange(n), np.zeros(n, np.int64), 1.35, None, "spectral")


def main():
    kernel, shower, cache = setup()
    route = ShowerTransport(kernel, ShowerData.of(str(cache), str(cache / "ge2-pack")))
    tables = route.tables()
    indices = _frequency_indices(route.kernel, route.config.frequency_nodes)
    bundle = tables["store"].bundle(route.kernel, indices)
    positions = np.asarray(kernel.detector.positions_m, float)

    moved, shift = moved_shower(shower, positions)
    response = route(moved)
    record = response.metadata["near_field"][0]
    near = near_field_ge2(route.kernel, moved, bundle, time_origin_ns=response.time_origin_ns)
    print("pass:", record["oms"], record["charge_pe"], record["elements"],
          int(response.active.sum()))

    edges = edge_elements(positions)
    rng = np.random.default_rng(3)
    origins = rng.uniform(-20.0, 40.0, len(positions))
    alone = near_field_ge2(route.kernel, edges, bundle, time_origin_ns=origins)
    print("edges:", alone.oms, alone.charge_pe[alone.oms], alone.metadata["elements"])

    def fields(el):
        return {name: np.asarray(getattr(el, name), float) for name in (
            "start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
            "start_ns", "end_ns")}

    out = dict(
        om=OM, gap_m=GAP_M, shift_m=shift,
        pass_charge_components_pe=response.charge_components_pe,
        pass_components_pe=response.components_pe.astype(np.float32),
        pass_spectrum_ge2_pe=response.spectrum_ge2_pe.astype(np.complex64),
        pass_time_origin_ns=response.time_origin_ns, pass_active=response.active,
        pass_ge2_charge_level=np.asarray(response.metadata["ge2_charge_level"], np.int8),
        pass_near_oms=np.asarray(record["oms"], np.int64),
        pass_near_charge_pe=np.asarray(record["charge_pe"], float),
        pass_near_elements=int(record["elements"]),
        pass_near_bins_added=np.asarray(record["bins_added_oms"], np.int64),
        pass_near_spectrum_pe=near.spectrum_pe[:, near.oms],
        edges_origins_ns=origins, edges_oms=np.asarray(alone.oms, np.int64),
        edges_charge_pe=alone.charge_pe[alone.oms],
        edges_spectrum_pe=alone.spectrum_pe[:, alone.oms],
        edges_elements=int(alone.metadata["elements"]),
        **{f"edges_{k}": v for k, v in fields(edges).items()})
    np.savez_compressed(Path(__file__).resolve().parent / "shower_near_c0.npz", **out)


if __name__ == "__main__":
    main()
