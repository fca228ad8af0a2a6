"""Oracle: order-0 direct light to the first glass entry (ctypes over ``order0.c``).

``candidates`` restates ``interval_candidates``
(``_ballistic_interval_numba.py:449-519``); ``rays`` restates the direct
first-entry quadrature ``_surface_ballistic_rays.evaluate``
(``_surface_ballistic_rays.py:36-156``), and ``direct_light`` repeats it with
the Gauss order doubled until every OM's charge and bins agree with the
previous order (``_surface_ballistic.py:149-168``, the ``adaptive`` loop).
Test infrastructure only.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .build import build

_LIB = None
_ERRORS = {-1: "point receiver lies on emitting track: singular ballistic fluence",
           -2: "emitting segment intersects the glass boundary",
           -3: "negative ballistic angular response", -4: "pair capacity exceeded"}


def _lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(str(build()))
        _LIB.o0_candidates.restype = C.c_int64
        _LIB.o0_rays.restype = C.c_int
    return _LIB


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def candidates(positions, radii, start, direction, length, c0, beta, phase_nodes, *,
               reach=np.inf, include_axis=True):
    positions, radii, start, direction = map(_f, (positions, radii, start, direction))
    length, c0, beta, phase_nodes = map(_f, (length, c0, beta, phase_nodes))
    cap = len(positions) * len(start)
    om = np.empty(max(cap, 1), np.int64)
    el = np.empty(max(cap, 1), np.int64)
    n = _lib().o0_candidates(len(positions), _p(positions), _p(radii), C.c_double(reach),
                             len(start), _p(start), _p(direction), _p(length), _p(c0), _p(beta),
                             len(phase_nodes), _p(phase_nodes), int(include_axis), _p(om), _p(el),
                             C.c_int64(cap))
    if n < 0:
        raise ValueError(_ERRORS[int(n)])
    return om[:n], el[:n]


def rays(pair_om, pair_element, det, el, optics, origins, edges, order):
    """Charge (OM,) and bins (OM, bins) at one Gauss order."""
    po = np.ascontiguousarray(pair_om, np.int64)
    pe = np.ascontiguousarray(pair_element, np.int64)
    n_om = len(det["positions_m"])
    edges, origins = _f(edges), _f(origins)
    charge = np.zeros(n_om)
    bins = np.zeros((n_om, len(edges) - 1))
    gx, gw = np.polynomial.legendre.leggauss(int(order))
    eff = _f(optics["efficiency_coefficients"])
    alpha = _f(det["alpha"])
    args = [_f(det["positions_m"]), _f(det["looks"]), _f(det["areas_m2"]), _f(det["radii_m"]),
            _f(el["start_m"]), _f(el["direction"]), _f(el["length_m"]), _f(el["coefficient0"]),
            _f(el["coefficient2"]), _f(el["beta"]), _f(el["start_ns"]), _f(el["end_ns"])]
    tabs = [_f(optics[k]) for k in ("panel_edges", "phase_nodes", "group_nodes",
                                    "extinction_nodes")]
    rc = _lib().o0_rays(C.c_int64(len(po)), _p(po), _p(pe), *map(_p, args),
                        len(tabs[0]), *map(_p, tabs), _p(eff), eff.shape[1], len(alpha), _p(alpha),
                        int(order), _p(gx), _p(gw), _p(origins), len(edges), _p(edges),
                        _p(charge), _p(bins))
    if rc:
        raise ValueError(_ERRORS[int(rc)])
    return charge, bins


def direct_light(pair_om, pair_element, det, el, optics, origins, edges, *, order=8,
                 max_order=64, relative_tolerance=2e-6, absolute_tolerance=1e-10,
                 bins_relative_tolerance=1e-4):
    """Order doubling per OM until charge (and bins L1) stop changing."""
    n_om = len(det["positions_m"])
    po = np.asarray(pair_om)
    q, b = rays(po, pair_element, det, el, optics, origins, edges, order)
    pending = np.ones(n_om, bool)
    while pending.any():
        order = min(2 * order, max_order)
        use = pending[po]
        x, y = rays(po[use], np.asarray(pair_element)[use], det, el, optics, origins, edges, order)
        dq = np.abs(x - q)
        db = np.abs(y - b).sum(axis=1)
        bad = pending & ((dq > absolute_tolerance + relative_tolerance * np.abs(x))
                         | (db > absolute_tolerance + bins_relative_tolerance * np.abs(x)))
        q[pending], b[pending] = x[pending], y[pending]
        if bad.any() and order == max_order:
            raise ValueError(f"ballistic rays quadrature failed for {int(bad.sum())} OMs at order {order}")
        pending = bad
    return q, b, order
