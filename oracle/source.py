"""Oracle: order >=2 sources of a shower on the band-fold node bands. Test infrastructure only.

Restates, in float64 NumPy, the shower route's source preparation:
* ``axis_frame``: ``AxisFrame.of`` (``axial_source.py:88-118``);
* ``compile_axial_slices`` (``_shower_basis.py:188-645``) with the route's
  ``ShowerBasis`` (``shower_basis.py:61-66``: 0.25 m slices, cubic axial
  weights, five-point transverse stencil of 0.2 m on the axis, thin-slice
  threshold 0.03 m, linear deposit on a 0.02 ns time lattice); the chord
  points' channels ``P_l(mu_C) Y_lm(u)`` (``_cone_harmonics``,
  ``_shower_basis.py:81-101``, ``_harmonics_into``,
  ``_directional_numba.py:90-128``) are summed per (slice, tick) row as one
  sparse product, then ``values = deposit @ exp(i tick omega)`` per slice;
* ``node_sources`` with ``_band_field`` (``shower/ge2.py:21-67``) and
  ``collapse`` (``:70-96``).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class AxialSource:
    """``AxialSource`` fields the route reads (``axial_source.py``)."""
    frame: tuple          # centre, axis, first, second
    z_m: np.ndarray
    transverse_m: np.ndarray
    channels: np.ndarray  # (points, nch, omega) complex
    reference_ns: float

    def points_m(self):
        centre, axis, first, second = self.frame
        return (centre[None, :] + self.z_m[:, None] * axis[None, :]
                + self.transverse_m[:, 0:1] * first[None, :]
                + self.transverse_m[:, 1:2] * second[None, :])


def axis_frame(el, photons):
    """``AxisFrame.of`` of elements with weights ``photons``."""
    points = el["start_m"] + 0.5 * el["length_m"][:, None] * el["direction"]
    weights = np.asarray(photons, float)
    share = weights / weights.sum()
    centre = (share[:, None] * points).sum(axis=0)
    offset = points - centre
    covariance = np.einsum("i,ij,ik->jk", share, offset, offset)
    values, vectors = np.linalg.eigh(covariance)
    if np.max(np.abs(values)) <= 1e-24:
        axis = np.sum(share[:, None] * el["direction"], axis=0)
        if np.linalg.norm(axis) <= 1e-12:
            _, angular = np.linalg.eigh(np.einsum("i,ij,ik->jk", share, el["direction"],
                                                  el["direction"]))
            axis = angular[:, -1]
    else:
        axis = vectors[:, int(np.argmax(values))]
    axis = axis / np.linalg.norm(axis)
    if float((share * (el["direction"] @ axis)).sum()) < 0:
        axis = -axis
    helper = np.array([0.0, 0.0, 1.0])
    if abs(float(axis @ helper)) > 0.9:
        helper = np.array([1.0, 0.0, 0.0])
    first = np.cross(axis, helper)
    first /= np.linalg.norm(first)
    return centre, axis, first, np.cross(axis, first)


def layout(degree, max_m):
    """``(starts, kept)`` of ``axial_fast._layout`` (``axial_fast.py:111-122``)."""
    starts, kept = [0], []
    for ell in range(degree + 1):
        for m in range(-min(ell, max_m), min(ell, max_m) + 1):
            kept.append(ell * ell + ell + m)
        starts.append(len(kept))
    return np.asarray(starts, np.int64), np.asarray(kept, np.int64)


def real_harmonics(x, y, z, degree):
    """Real orthonormal harmonics of unit vectors (rows), flat ``l*l+l+m``
    (``_harmonics_into``, ``_directional_numba.py:90-128``), vectorised over rows."""
    n = len(x)
    out = np.zeros((n, (degree + 1) ** 2))
    radius = np.sqrt(x * x + y * y + z * z)
    mu = z / radius
    transverse = np.sqrt(x * x + y * y)
    sine = transverse / radius
    zero = transverse == 0.0
    safe = np.where(zero, 1.0, transverse)
    cp = np.where(zero, 1.0, x / safe)
    sp = np.where(zero, 0.0, y / safe)
    cm, sm = np.ones(n), np.zeros(n)
    diagonal = np.full(n, 1.0 / np.sqrt(4 * np.pi))
    for m in range(degree + 1):
        if m:
            diagonal = diagonal * (np.sqrt((2.0 * m + 1) / (2.0 * m)) * sine)
            cm, sm = cm * cp - sm * sp, sm * cp + cm * sp
        v0 = diagonal
        v1 = None
        for ell in range(m, degree + 1):
            if ell == m:
                value = v0
            elif ell == m + 1:
                value = np.sqrt(2 * m + 3) * mu * v0
                v1 = value
            else:
                aa = np.sqrt((4.0 * ell * ell - 1) / (ell * ell - m * m))
                bb = np.sqrt(((2.0 * ell + 1) * ((ell - 1) ** 2 - m * m))
                             / ((2.0 * ell - 3) * (ell * ell - m * m)))
                value = aa * mu * v1 - bb * v0
                v0 = v1
                v1 = value
            centre = ell * ell + ell
            if m == 0:
                out[:, centre] = value
            else:
                out[:, centre - m] = np.sqrt(2) * value * sm
                out[:, centre + m] = np.sqrt(2) * value * cm
    return out


def cone_harmonics(vectors, cones, degree, starts, kept):
    """``P_l(mu_C) Y_lm(u)`` of every element on the kept channels."""
    full = real_harmonics(vectors[:, 0], vectors[:, 1], vectors[:, 2], degree)[:, kept]
    prev = np.ones(len(cones))
    current = np.asarray(cones, float)
    for ell in range(degree + 1):
        if ell == 0:
            p = np.ones(len(cones))
        elif ell == 1:
            p = current
        else:
            p = ((2 * ell - 1) * cones * current - (ell - 1) * prev) / ell
            prev, current = current, p
        full[:, starts[ell]:starts[ell + 1]] *= p[:, None]
    return full


def axial_weights(r):
    """Cubic Lagrange slice shifts and weights (``_shower_basis.py:129-135``)."""
    return ((-1, 0, 1, 2),
            (-r * (r - 1) * (r - 2) / 6, (r + 1) * (r - 1) * (r - 2) / 2,
             -(r + 1) * r * (r - 2) / 2, (r + 1) * r * (r - 1) / 6))


def compile_axial_slices(el, photons, cones, degree, omega, frame, *, azimuthal_degree,
                         cell_m=0.25, stencil_m=0.2, stencil_threshold_m=0.03,
                         time_step_ns=0.02):
    """One field's axial-slice source (stencil on the axis, linear time deposit)."""
    from scipy import sparse
    centre, axis, first, second = (np.asarray(v, float) for v in frame)
    omega = np.atleast_1d(np.asarray(omega, float))
    charge_only = len(omega) == 1 and omega[0] == 0
    photons = np.asarray(photons, float)
    count = len(photons)
    max_m = min(int(degree), int(azimuthal_degree))
    starts, kept = layout(int(degree), max_m)
    nch = len(kept)
    element_order = 1 if float(np.max(el["length_m"])) <= cell_m / 10 else 2
    nodes, node_weights = np.polynomial.legendre.leggauss(element_order)
    nodes, node_weights = (nodes + 1) / 2, node_weights / 2
    reference = float(np.asarray(el["start_ns"]).min())

    def coordinates(fraction):
        points = el["start_m"] + (fraction * el["length_m"])[:, None] * el["direction"]
        offset = points - centre
        z = offset @ axis
        transverse = offset - z[:, None] * axis
        time = el["start_ns"] + fraction * (el["end_ns"] - el["start_ns"])
        return z, transverse, time

    z_origin = float(coordinates(0.5)[0].min()) - 2 * cell_m
    coords = [coordinates(f) for f in nodes]
    time_max = max(float(np.max(c[2])) for c in coords)
    kmax = 1 if charge_only else int(np.floor((time_max - reference) / time_step_ns)) + 3
    ticks = 1 if charge_only else 2
    links = ticks * 4
    keys, link_weights, factors, geometry_links = [], [], [], []
    for (z, offset, time), node_weight in zip(coords, node_weights):
        x = offset @ first
        y = offset @ second
        mom = np.stack([np.ones(count), x, y, x * x, y * y], axis=1)
        factors.append(photons[:, None] * mom * node_weight)
        zl = (z - z_origin) / cell_m
        zb = np.floor(zl).astype(np.int64)
        if charge_only:
            tb = np.zeros(count, np.int64)
            tick_weights = ((0, 1.0),)
        else:
            tl = (np.asarray(time, float) - reference) / time_step_ns
            tb = np.floor(tl).astype(np.int64)
            tr = tl - tb
            tick_weights = ((0, 1 - tr), (1, tr))
        shifts, zw = axial_weights(zl - zb)
        geometry_links.append([(zb + shift, wz) for shift, wz in zip(shifts, zw)])
        key = np.empty((count, links), np.int64)
        weight = np.empty((count, links))
        j = 0
        for shift, wz in zip(shifts, zw):
            for dt, wt in tick_weights:
                key[:, j] = (zb + shift) * kmax + tb + dt
                weight[:, j] = wz * wt
                j += 1
        keys.append(key)
        link_weights.append(weight)
    keys = np.concatenate(keys, axis=1)
    unique, inverse = np.unique(keys, return_inverse=True)
    rows = np.asarray(inverse).reshape(count, -1).astype(np.int64)
    cell_of = unique // kmax
    tick_of = unique % kmax
    slices, row_start = np.unique(cell_of, return_index=True)
    row_start = np.append(row_start, len(unique)).astype(np.int64)
    zero = np.zeros((len(slices), 5))
    for links_n, factor in zip(geometry_links, factors):
        for cell_ids, weight in links_n:
            rows_n = np.searchsorted(slices, cell_ids)
            for moment in range(5):
                zero[:, moment] += np.bincount(rows_n, weights=weight * factor[:, moment],
                                               minlength=len(slices))
    mass = zero[:, 0]
    safe = np.where(np.abs(mass) > 0, mass, 1.0)
    spread = np.sqrt(np.abs(zero[:, 3] + zero[:, 4]) / np.abs(safe))
    wide = spread > stencil_threshold_m
    centroid = np.stack([np.where(wide, 0.0, zero[:, 1] / safe),
                         np.where(wide, 0.0, zero[:, 2] / safe)], axis=1)
    z_centres = z_origin + slices * cell_m
    h = float(stencil_m)
    wide_index = np.cumsum(wide) - 1
    count_wide = int(wide.sum())
    npoints = len(slices) + 4 * count_wide
    # deposit[row, moment, channel] = sum over chord points and links of
    # weight * factor[moment] * harmonic[channel]
    vectors = np.stack((el["direction"] @ first, el["direction"] @ second,
                        el["direction"] @ axis), axis=-1)
    harmonics = cone_harmonics(vectors, np.asarray(cones, float), int(degree), starts, kept)
    deposit = np.zeros((len(unique), 5 * nch))
    for n in range(len(nodes)):
        span = slice(n * links, (n + 1) * links)
        block = (factors[n][:, :, None] * harmonics[:, None, :]).reshape(count, 5 * nch)
        matrix = sparse.csr_matrix(
            (link_weights[n].ravel(), (rows[:, span].ravel(),
                                       np.repeat(np.arange(count), links))),
            shape=(len(unique), count))
        deposit += matrix @ block
    deposit = deposit.reshape(len(unique), 5, nch)
    table = np.zeros((npoints, nch, len(omega)), complex)
    times = tick_of * time_step_ns
    for cell in range(len(slices)):
        span = slice(row_start[cell], row_start[cell + 1])
        keep = [0, 1, 2, 3, 4] if wide[cell] else [0]
        phase = np.outer(times[span], omega)
        blk = deposit[span][:, keep].reshape(-1, len(keep) * nch).T
        values = ((blk @ np.cos(phase)) + 1j * (blk @ np.sin(phase))).reshape(
            len(keep), nch, len(omega))
        if not wide[cell]:
            table[cell] = values[0]
            continue
        m0, mx, my, mxx, myy = values
        ids = [cell] + [len(slices) + offset * count_wide + wide_index[cell] for offset in range(4)]
        for point, value in zip(ids, [m0 - (mxx + myy) / h ** 2, 0.5 * (mxx / h ** 2 + mx / h),
                                      0.5 * (mxx / h ** 2 - mx / h), 0.5 * (myy / h ** 2 + my / h),
                                      0.5 * (myy / h ** 2 - my / h)]):
            table[point] = value
    offsets = [(h, 0.0), (-h, 0.0), (0.0, h), (0.0, -h)]
    points_z = np.concatenate([z_centres] + [z_centres[wide]] * 4)
    points_t = np.concatenate([centroid] + [np.tile(o, (count_wide, 1)) for o in offsets])
    return AxialSource((centre, axis, first, second), points_z, points_t, table, reference)


def band_field(el, wavelength_nm, phase_index):
    """``_band_field`` (``shower/ge2.py:21-32``): elements above this band's
    threshold, photons ``c0 / l^2 + c2 / (l^2 n^2)``, cone ``1 / (beta n)``."""
    mask = el["beta"] * phase_index > 1
    if not np.any(mask):
        return None
    sub = el if np.all(mask) else {k: v[mask] for k, v in el.items()}
    scale0 = 1.0 / wavelength_nm ** 2
    scale2 = scale0 / phase_index ** 2
    photons = scale0 * sub["coefficient0"] - scale2 * (-sub["coefficient2"])
    return sub, photons, 1.0 / (sub["beta"] * phase_index)


def node_sources(el, wavelengths, phases, scales, bands, degree, azimuthal_degree, omega, frame):
    """``node_sources`` (``shower/ge2.py:35-67``): one compile per node band,
    scaled by the fold scale; a band without emitting elements takes another
    band's points with zero channels."""
    compiled = {}
    for band in bands:
        field = band_field(el, float(wavelengths[band]), float(phases[band]))
        if field is None:
            continue
        sub, photons, cones = field
        compiled[band] = compile_axial_slices(sub, photons, cones, degree, omega, frame,
                                              azimuthal_degree=azimuthal_degree)
    if not compiled:
        raise ValueError("no element emits in any node band")
    template = next(iter(compiled.values()))
    out = []
    for band in bands:
        item = compiled.get(band)
        if item is None:
            item = AxialSource(template.frame, template.z_m, template.transverse_m,
                               np.zeros_like(template.channels), template.reference_ns)
        out.append(AxialSource(item.frame, item.z_m, item.transverse_m,
                               item.channels * float(scales[band]), item.reference_ns))
    return out


def collapse(sources, cell_m):
    """``collapse`` (``shower/ge2.py:70-96``): zero-frequency channels summed per
    ``cell_m`` cube of the frame at the |l=0|-weighted centroid."""
    reduced = []
    for item in sources:
        weight = np.abs(item.channels[:, 0, 0])
        coordinates = np.column_stack((item.z_m, item.transverse_m))
        keys = np.floor(coordinates / float(cell_m)).astype(np.int64)
        _, inverse = np.unique(keys, axis=0, return_inverse=True)
        inverse = np.asarray(inverse).ravel()
        chunks = [np.flatnonzero(inverse == group) for group in range(int(inverse.max()) + 1)]
        z, transverse, channels = [], [], []
        for chunk in chunks:
            total = weight[chunk].sum()
            share = (weight[chunk] / total if total > 0 else np.full(len(chunk), 1.0 / len(chunk)))
            z.append(np.sum(share * item.z_m[chunk]))
            transverse.append(share @ item.transverse_m[chunk])
            channels.append(item.channels[chunk, :, :1].sum(axis=0))
        reduced.append(AxialSource(item.frame, np.asarray(z), np.asarray(transverse),
                                   np.ascontiguousarray(np.asarray(channels)), item.reference_ns))
    return reduced
