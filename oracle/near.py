"""Oracle: the near-field clamp of order >=2 (test infrastructure only).

Restates ``near_field_ge2`` (``near_field.py:91-171``) with ``near_portions``
(``:39-69``, a brute-force distance test in place of the k-d tree: the same
portions, since a chord within the radius lies within half a length of the
element midpoint), ``_harmonics`` (``:72-88``) and the clamped fused-looks
evaluator ``_cone_many_looks`` with ``clamp_low = 0``
(``muon/track_ge2_primitive.py:612-660``) for one look, in float64 NumPy. The
splines are the first radial interval of every wavelength's order >=2 spline
(``tables/near_<config>.npz``); every near point takes that interval (its
amplitude radius is the radial minimum), so no other interval is needed.
"""
import numpy as np
from scipy.special import eval_legendre

from .ge2 import harmonics, start_norm_table, wigner


def near_portions(positions, el, radius):
    """``{om: [(element, s0, s1), ...]}`` in element order (``near_field.py:39-69``)."""
    start, direction, length = el["start_m"], el["direction"], el["length_m"]
    portions = {}
    for index in range(len(length)):
        delta = positions - start[index]
        z = delta @ direction[index]
        rho2 = np.maximum(np.einsum("ij,ij->i", delta, delta) - z * z, 0.0)
        for om in np.flatnonzero(rho2 < radius * radius):
            half = np.sqrt(radius * radius - rho2[om])
            s0, s1 = max(z[om] - half, 0.0), min(z[om] + half, float(length[index]))
            if s1 > s0:
                portions.setdefault(int(om), []).append((index, s0, s1))
    return dict(sorted(portions.items()))


def cone_harmonics(el, index, wavelength_nm, phase_index, degree):
    """Spectral cone harmonics per unit coefficient0 (``near_field.py:72-88``)."""
    ell = np.arange(degree + 1)
    norm = np.sqrt((2 * ell + 1) / (4 * np.pi))
    c0 = float(el["coefficient0"][index])
    ratio = float(el["coefficient2"][index] / c0) if c0 > 0 else 0.0
    beta = float(el["beta"][index])
    out = np.zeros((len(wavelength_nm), degree + 1))
    for band, (wavelength, phase) in enumerate(zip(wavelength_nm, phase_index)):
        yield_ = (1 + ratio / phase ** 2) / wavelength ** 2
        if beta * phase <= 1 or yield_ <= 0:
            continue
        out[band] = norm * eval_legendre(ell, 1 / (beta * phase)) * yield_
    return out


def clamped_point(table, impact, u, look, h, weights, alpha):
    """``_cone_many_looks`` for one point and one look with ``clamp_low = 0``:
    the (frequency,) spectrum per unit coefficient0 (``:628-659``)."""
    coef = table["coefficients"]                         # (lam, l, pair, 4, w)
    log_r, omega = table["log_r"], table["omega"]
    degree, max_out = int(table["degree"]), int(table["acceptance_degree"])
    pair_lambda, pair_mu = table["pair_lambda"], table["pair_mu"]
    radius = np.hypot(impact, u)
    if radius > table["radial_high_m"] or radius == 0.0:
        return np.zeros(len(omega), complex)
    cosine, sine = u / radius, impact / radius
    wig = wigner(degree, max_out, 0, cosine, start_norm_table(max_out), max_out)
    amplitude = max(radius, float(np.exp(log_r[0])))
    t = np.log(amplitude) - log_r[0]
    scale = weights * np.exp(-table["absorption"] * amplitude) / (4 * np.pi * amplitude ** 2)
    phase = scale[:, None] * np.exp(1j * np.outer(1.0 / table["speed"], omega) * radius)
    radial = ((coef[..., 0, :] * t + coef[..., 1, :]) * t + coef[..., 2, :]) * t + coef[..., 3, :]
    lx, ly, lz = look
    detector = harmonics(cosine * lx - sine * lz, ly, sine * lx + cosine * lz, max_out)
    result = np.zeros(len(omega), complex)
    for p, (lam, mu) in enumerate(zip(pair_lambda, pair_mu)):
        factor = alpha[lam] * detector[lam * lam + lam + mu]
        for ell in range(mu, degree + 1):
            rotation = wig[ell, max_out, 0] if mu == 0 else \
                np.sqrt(2.0) * (-1.0) ** mu * wig[ell, max_out + mu, 0]
            result += factor * rotation * np.sum(h[:, ell, None] * radial[:, ell, p]
                                                 * phase, axis=0)
    return result


def near_field(table, el, positions, looks, areas, origins, *, wavelength_nm, weight_nm,
               efficiency, phase_index, alpha, panel_m=0.05, gauss_order=6, radius=None):
    """``near_field_ge2``: (oms, charge (OM,), spectrum (frequency, OM), evaluated
    portions) for elements ``el`` (the reference's field names) and OMs whose
    ``looks`` are ``-orientations``."""
    omega = np.asarray(table["omega"], float)
    degree = int(table["degree"])
    radius = float(np.exp(table["log_r"][0])) if radius is None else float(radius)
    nodes, gauss = np.polynomial.legendre.leggauss(int(gauss_order))
    n = len(positions)
    charge = np.zeros(n)
    spectrum = np.zeros((len(omega), n), complex)
    portions = near_portions(positions, el, radius)
    evaluated = 0
    for om, parts in portions.items():
        weights = np.asarray(weight_nm) * np.asarray(efficiency) * float(areas[om])
        for index, s0, s1 in parts:
            axis = el["direction"][index]
            delta = positions[om] - el["start_m"][index]
            z = float(delta @ axis)
            radial = delta - z * axis
            rho = float(np.linalg.norm(radial))
            if rho < 1e-9:
                trial = np.array([1., 0., 0.]) if abs(axis[0]) < .9 else np.array([0., 1., 0.])
                radial = trial - (trial @ axis) * axis
                rho = 1e-9
            ex = radial / np.linalg.norm(radial)
            ey = np.cross(axis, ex)
            look = np.array([looks[om] @ ex, looks[om] @ ey, looks[om] @ axis])
            h = cone_harmonics(el, index, wavelength_nm, phase_index, degree)
            if not np.any(h):
                continue
            count = max(1, int(np.ceil((s1 - s0) / panel_m)))
            edges = np.linspace(z - s1, z - s0, count + 1)
            half = np.diff(edges) / 2
            u = (edges[:-1, None] + half[:, None] * (nodes + 1)).ravel()
            w = (half[:, None] * gauss).ravel()
            values = np.array([clamped_point(table, rho, x, look, h, weights, alpha) for x in u])
            length = float(el["length_m"][index])
            clock = float(el["end_ns"][index] - el["start_ns"][index]) / length
            density = float(el["coefficient0"][index]) / length
            closest = float(el["start_ns"][index]) + z * clock - origins[om]
            part = density * np.exp(1j * omega * closest) * (
                (w[:, None] * values * np.exp(-1j * u[:, None] * clock * omega)).sum(0))
            spectrum[:, om] += part
            charge[om] += part[0].real
            evaluated += 1
    return np.array(sorted(portions), int), charge, spectrum, evaluated
