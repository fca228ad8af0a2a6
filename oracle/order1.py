"""Oracle: grouped-pencil order 1 (ctypes over ``order1.c``). Test infrastructure only.

``compress`` restates stage A (``prompt.py:1317-1402``; with ``parent_face``
also ``compress_screen``/``pack_pencils``, ``_prompt_screen.py:44-98``);
``grouped`` restates ``grouped_pencils_order1`` (``_prompt_numba.py:1750-2064``)
and, for a screen pack, ``screen_order1`` (``_prompt_screen.py:172-503``).
``oracle.shower`` runs them as the reference's fused-band order 1 with its
global coarse screen (``prompt.py:720-812``).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from .build import build

_LIB = None
FIELDS = (("position", 3), ("direction", 3), ("w0", 1), ("w2", 1), ("time", 1), ("major", 3),
          ("var_major", 1), ("var_minor", 1), ("pos_cov", 6))
# _IFUNC_TAYLOR (_prompt_numba.py:132-135)
TAYLOR = np.asarray([[1.0 / (math.factorial(n) * (n + j + 1.0)) for n in range(24)]
                     for j in range(3)], dtype=np.float64)
_GL48 = np.polynomial.legendre.leggauss(48)
GAUSS_TAU = 0.25 * math.pi * (_GL48[0] + 1.0)
GAUSS_W = 0.25 * math.pi * _GL48[1]
# _prepare_gauss_inverse (_prompt_numba.py:103-112)
GAUSS_TANGENT = np.array([math.tan(t) for t in GAUSS_TAU])
GAUSS_WSEC2 = np.array([w * (1.0 + t * t) for w, t in zip(GAUSS_W, GAUSS_TANGENT)])


def _lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(str(build()))
        _LIB.o1c_compress.restype = C.c_void_p
        _LIB.o1c_count.restype = C.c_int64
        _LIB.o1c_count.argtypes = [C.c_void_p, C.c_int]
        _LIB.o1c_ring_nodes.restype = C.c_int64
        _LIB.o1c_ring_nodes.argtypes = [C.c_void_p]
        _LIB.o1c_fetch.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 11
        _LIB.o1c_free.argtypes = [C.c_void_p]
        _LIB.o1c_grouped.restype = C.c_int
    return _LIB


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def _field(el, name):
    return np.asarray(el[name] if isinstance(el, dict) else getattr(el, name), float)


def compress(elements, cone_cos, *, cell_m=0.5, pixel_face=96, ring_nodes=192, parent_face=0):
    """Stage A pencils (and, with ``parent_face``, the coarse screen's preorder
    pack with ``hierarchy_parent`` / ``next_node``)."""
    start = _f(_field(elements, "start_m"))
    direction = _f(_field(elements, "direction"))
    length = _f(_field(elements, "length_m"))
    ends = start + length[:, None] * direction
    low = np.minimum(start.min(axis=0), ends.min(axis=0)) - cell_m
    high = np.maximum(start.max(axis=0), ends.max(axis=0)) + cell_m
    dims = _i(np.ceil((high - low) / cell_m).astype(np.int64) + 1)
    if float(np.prod(dims.astype(float))) * 6 * int(pixel_face) ** 2 >= 2.0 ** 62:
        raise ValueError("cell grid too large for 64-bit pencil keys; increase cell_m")
    arrays = [start, direction, length, _f(_field(elements, "coefficient0")),
              _f(_field(elements, "coefficient2")), _f(cone_cos), _f(_field(elements, "start_ns")),
              _f(_field(elements, "end_ns"))]
    lib = _lib()
    h = lib.o1c_compress(C.c_int64(len(length)), *[_p(a) for a in arrays], C.c_double(cell_m),
                         C.c_int(int(pixel_face)), C.c_int(int(ring_nodes)), _p(_f(low)), _p(dims),
                         C.c_int(int(parent_face)))
    if not h:
        raise MemoryError("oracle compress failed")
    try:
        out = []
        for which in ((0, 1) if parent_face else (0,)):
            n = int(lib.o1c_count(h, which))
            t = {k: np.empty((n, w) if w > 1 else n) for k, w in FIELDS}
            parent = np.empty(n, np.int64) if which else None
            nxt = np.empty(n, np.int64) if which else None
            lib.o1c_fetch(h, which, *[_p(t[k]) for k, _ in FIELDS], _p(parent), _p(nxt))
            if which:
                t["hierarchy_parent"], t["next_node"] = parent, nxt
            t["ring_nodes_deposited"] = int(lib.o1c_ring_nodes(h))
            out.append(t)
    finally:
        lib.o1c_free(h)
    return out[0] if not parent_face else (out[0], out[1])


def grouped(pencils, receivers, looks, areas, origins, work, monomials, g, bands, edges, *,
            path_step=0.1, path_step_tail=0.25, tail_exponent=25.0, direct_bins=4,
            max_path_nodes=2048, smoothing_factor=6.0, merge=(2e-3, 0.08, 0.5, 0.02),
            compute_bins=True):
    """``grouped_pencils_order1`` for the OMs ``work`` (``screen_order1`` when
    the pencils carry a hierarchy). ``bands``: ``mus, mut, speed, s0w, s2w``.
    Returns ``(charge, bins, groups, batches)`` per OM."""
    coef, ipow, jpow, degree = monomials
    receivers, looks = _f(receivers), _f(looks)
    n = len(receivers)
    areas = _f(np.broadcast_to(np.asarray(areas, float), (n,)))
    origins = _f(origins)
    work = _i(work)
    edges = _f(edges)
    mus, mut, speed, s0w, s2w = (_f(bands[k]) for k in ("mus", "mut", "speed", "s0w", "s2w"))
    kappa = -mut * speed
    eedge = _f(np.exp(np.outer(kappa, edges)))
    width = np.diff(edges)
    itab = np.empty((len(kappa), len(width), 3))
    for lam, value in enumerate(kappa):  # interval_table (_prompt_numba.py:635-644)
        for k, w in enumerate(width):
            z = value * w
            ez = math.exp(z)
            if abs(z) < 1.0:
                i0, i1, i2 = TAYLOR[0, 23], TAYLOR[1, 23], TAYLOR[2, 23]
                for m in range(22, -1, -1):
                    i0, i1, i2 = i0 * z + TAYLOR[0, m], i1 * z + TAYLOR[1, m], i2 * z + TAYLOR[2, m]
            else:
                i0 = (ez - 1.0) / z
                i1 = (ez * (z - 1.0) + 1.0) / (z * z)
                i2 = (ez * (z * z - 2.0 * z + 2.0) - 2.0) / (z * z * z)
            itab[lam, k] = (i0, i1, i2)
    y_g = (1.0 - abs(g)) / (1.0 + abs(g)) if g != 0 else 1.0
    screen = "hierarchy_parent" in pencils
    nb = len(edges) - 1
    charge = np.zeros(n)
    bins = np.zeros((n, nb if compute_bins else 0))
    groups = np.zeros(n, np.int64)
    batches = np.zeros(n, np.int64)
    P = {k: _f(pencils[k]) for k, _ in FIELDS}
    parent = _i(pencils["hierarchy_parent"]) if screen else None
    nxt = _i(pencils["next_node"]) if screen else None
    theta_lo, theta_ratio, tau_step, log_r_step = (float(v) for v in merge)
    rc = _lib().o1c_grouped(
        C.c_int64(n), _p(receivers), _p(looks), _p(areas), _p(origins), C.c_int64(len(work)),
        _p(work), C.c_int64(len(P["w0"])), *[_p(P[k]) for k, _ in FIELDS], _p(parent), _p(nxt),
        C.c_int(len(GAUSS_TANGENT)), _p(GAUSS_TANGENT), _p(GAUSS_WSEC2), _p(TAYLOR),
        C.c_int(len(coef)), _p(_f(coef)), _p(_i(ipow)), _p(_i(jpow)), C.c_int(int(degree)),
        C.c_double(g), C.c_double(y_g), C.c_double(path_step), C.c_double(path_step_tail),
        C.c_double(tail_exponent), C.c_int(len(mus)), _p(mus), _p(mut), _p(speed), _p(s0w),
        _p(s2w), C.c_int(len(edges)), _p(edges), _p(eedge), _p(_f(itab)), C.c_int(direct_bins),
        C.c_int(max_path_nodes), C.c_double(smoothing_factor), C.c_double(theta_lo),
        C.c_double(theta_ratio), C.c_double(tau_step), C.c_double(log_r_step),
        C.c_double(float(np.max(speed))), C.c_int(int(bool(compute_bins))), _p(charge),
        _p(bins) if compute_bins else None, _p(groups), _p(batches))
    if rc:
        raise MemoryError("oracle grouped order 1: scratch allocation failed")
    return charge, bins, groups, batches


def acceptance_monomials(alpha):
    """``(coef, ipow, jpow, degree)`` of the Legendre acceptance in ``c1, c3``
    (``acceptance_monomials``, ``prompt.py:380-399``)."""
    from math import comb
    alpha = np.asarray(alpha, float)
    series = alpha * (2 * np.arange(len(alpha)) + 1) / (4 * np.pi)
    power = np.polynomial.legendre.leg2poly(series)
    degree = len(power) - 1
    coef, ipow, jpow = [], [], []
    for k in range(degree + 1):
        for i in range(k + 1):
            coef.append(power[k] * comb(k, i))
            ipow.append(i)
            jpow.append(k - i)
    return np.asarray(coef, float), np.asarray(ipow), np.asarray(jpow), int(degree)


SCREEN = dict(cell_m=2.0, pixel_face=8, ring_nodes=24, refine_factor=4)  # prompt.py:182-185


def screen_pencils(elements, cone_cos):
    """``compress_screen`` (``_prompt_screen.py:91-98``): 2 m cells, 32-pixel
    faces under 8-pixel parents, 24 ring nodes."""
    _, pack = compress(elements, cone_cos, cell_m=SCREEN["cell_m"],
                       pixel_face=SCREEN["pixel_face"] * SCREEN["refine_factor"],
                       ring_nodes=SCREEN["ring_nodes"], parent_face=SCREEN["pixel_face"])
    return pack
