"""Not-a-knot cubic splines as explicit linear operators (host, float64).

The reference interpolates with SciPy's ``CubicSpline`` (default not-a-knot
boundary) in two places on this path: the radial lookup of the multipole
tables in log r (``cache.py:334``) and the 65 -> 321 frequency refinement of
the readout (``readout.py:60-62``, ``shower/api.py:559-565``). A cubic spline
is linear in its data, so both become matrices built once on the host: the
per-interval polynomial coefficients as a map from the knot values, and the
resampling onto a finer grid as a dense (new, old) matrix.

The construction is the textbook first-derivative formulation: interior
rows enforce continuity of the second derivative,
``h_i s_{i-1} + 2 (h_{i-1} + h_i) s_i + h_{i-1} s_{i+1} = 3 (h_i d_{i-1} + h_{i-1} d_i)``
with ``d_i`` the secant slopes, and the two end rows enforce continuity of
the third derivative at the second and second-to-last knots. It is solved
densely (a few hundred knots at most).
"""
from __future__ import annotations

import numpy as np

__all__ = ["slope_operator", "coefficient_operator", "resample_matrix", "spline_coefficients"]


def slope_operator(x):
    """Matrix ``G`` (n, n) with knot slopes ``s = G @ y`` of the not-a-knot spline."""
    x = np.asarray(x, float)
    n = len(x)
    if n < 4:
        raise ValueError("not-a-knot splines here need at least four knots")
    h = np.diff(x)
    # secant slopes d_i = D @ y
    D = np.zeros((n - 1, n))
    D[np.arange(n - 1), np.arange(n - 1)] = -1.0 / h
    D[np.arange(n - 1), np.arange(1, n)] = 1.0 / h
    A = np.zeros((n, n))
    R = np.zeros((n, n - 1))
    for i in range(1, n - 1):
        A[i, i - 1] = h[i]
        A[i, i] = 2 * (h[i - 1] + h[i])
        A[i, i + 1] = h[i - 1]
        R[i, i - 1] = 3 * h[i]
        R[i, i] = 3 * h[i - 1]
    # not-a-knot at x_1: third derivative continuous across the first interior knot
    A[0, 0] = h[1]
    A[0, 1] = h[0] + h[1]
    R[0, 0] = ((h[0] + 2 * (h[0] + h[1])) * h[1]) / (h[0] + h[1])
    R[0, 1] = h[0] ** 2 / (h[0] + h[1])
    # not-a-knot at x_{n-2}
    A[n - 1, n - 2] = h[-1] + h[-2]
    A[n - 1, n - 1] = h[-2]
    R[n - 1, n - 3] = h[-1] ** 2 / (h[-2] + h[-1])
    R[n - 1, n - 2] = ((2 * (h[-2] + h[-1]) + h[-1]) * h[-2]) / (h[-2] + h[-1])
    return np.linalg.solve(A, R @ D)


def coefficient_operator(x):
    """Tensor ``C`` (n-1, 4, n): interval polynomial coefficients ``C @ y``.

    On interval ``i`` with ``t = x - x_i`` the spline is
    ``c0 t^3 + c1 t^2 + c2 t + c3`` (highest power first).
    """
    x = np.asarray(x, float)
    n = len(x)
    h = np.diff(x)
    G = slope_operator(x)
    eye = np.eye(n)
    C = np.zeros((n - 1, 4, n))
    for i in range(n - 1):
        d = (eye[i + 1] - eye[i]) / h[i]
        s0, s1 = G[i], G[i + 1]
        tt = (s0 + s1 - 2 * d) / h[i]
        C[i, 0] = tt / h[i]
        C[i, 1] = (d - s0) / h[i] - tt
        C[i, 2] = s0
        C[i, 3] = eye[i]
    return C


def spline_coefficients(x, y, axis=0):
    """Interval coefficients of the not-a-knot spline of ``y`` along ``axis``.

    Returns an array with the knot axis replaced by (interval, 4) at the same
    position (highest power first), in the dtype of ``y`` (real or complex).
    """
    y = np.moveaxis(np.asarray(y), axis, 0)
    C = coefficient_operator(x)
    out = np.tensordot(C, y, axes=([2], [0]))  # (n-1, 4, ...)
    return np.moveaxis(out, [0, 1], [axis, axis + 1])


def _interval(x, xnew):
    """SciPy's interval rule: ``searchsorted(x, xnew, 'right') - 1`` clipped."""
    j = np.searchsorted(x, xnew, side="right") - 1
    return np.clip(j, 0, len(x) - 2)


def resample_matrix(x, xnew):
    """Dense matrix ``S`` (len(xnew), len(x)) with ``spline(x, y)(xnew) = S @ y``."""
    x = np.asarray(x, float)
    xnew = np.asarray(xnew, float)
    C = coefficient_operator(x)
    j = _interval(x, xnew)
    t = xnew - x[j]
    powers = np.stack([t ** 3, t ** 2, t, np.ones_like(t)], axis=1)  # (m, 4)
    return np.einsum("mp,mpn->mn", powers, C[j])
