"""Oracle: isotropic calibration flash, all orders (reference ``transport.py``).

Restates ``TransportKernel._transport_isotropic`` (``transport.py:1061-1164``)
for a monochromatic flash read by the centre-ray receiver, with the multipole
lookup of ``ResponseCache.moments_at`` (``cache.py:294-336``) and
``ResponseCache.acceptance_spectrum`` (``cache.py:372-436``). Float64 NumPy;
the cubic spline in log r is SciPy's not-a-knot ``CubicSpline`` as in
``cache.py:334``.
"""
import numpy as np
from scipy.interpolate import CubicSpline
from scipy.special import eval_legendre

from .readout import readout_bins

C_VACUUM_M_PER_NS = 0.299792458


def acceptance_from_alpha(alpha, cosines, tolerance=1e-12):
    """``cache.py:509-521``: A(x) = sum_l alpha_l (2l+1) P_l(x) / (4 pi)."""
    alpha = np.asarray(alpha, float)
    peak = np.max(np.abs(alpha))
    significant = np.flatnonzero(np.abs(alpha) > tolerance * peak) if peak > 0 else []
    top = int(significant[-1]) if len(significant) else 0
    ell = np.arange(top + 1)
    basis = eval_legendre(ell[None, :], np.atleast_1d(cosines)[:, None])
    return basis @ (alpha[:top + 1] * (2 * ell + 1)) / (4 * np.pi)


def moments_at(table, radii, top):
    """``cache.py:294-336``: spline of detrended moments in log r, flight phase."""
    omega = np.asarray(table["omega_per_ns"], float)
    grid_r = np.asarray(table["radii_m"], float)
    mu_a = float(table["absorption_per_m"])
    speed = C_VACUUM_M_PER_NS / float(table["group_index"])

    def scale(r):
        return np.exp(-mu_a * r) / (4 * np.pi * r ** 2)

    flight = str(table["radial_phase"]) == "flight"
    key = ("_spline", top)
    spline = table.get(key)
    if spline is None:  # the reference caches the spline per degree count too (cache.py:321-334)
        block = np.asarray(table["moments"])[:, :, :top]
        detrended = block / scale(grid_r)[None, :, None, None]
        if flight:
            detrended = detrended * np.exp(
                -1j * omega[:, None] * grid_r[None, :] / speed)[:, :, None, None]
        spline = table[key] = CubicSpline(np.log(grid_r), detrended, axis=1)
    out = spline(np.log(radii)) * scale(radii)[None, :, None, None]
    if flight:
        out = out * np.exp(1j * omega[:, None] * radii[None, :] / speed)[:, :, None, None]
    return out


def transport_flash(table, detector, flash, config):
    """One monochromatic isotropic flash; returns the response arrays.

    ``detector``: dict with ``positions_m`` (D,3), ``orientations`` (D,3),
    ``area_m2`` (D,), ``alpha`` (Legendre coefficients of the acceptance up
    to the table degree), ``acceptance`` (callable, optional; else rebuilt
    from ``alpha``), ``spectral_weight`` (efficiency at the flash wavelength).
    ``flash``: dict with ``position_m``, ``photons``, ``time_ns``.
    ``config``: dict with ``omega_per_ns``, ``readout_omega_per_ns``,
    ``edges_ns``, ``threshold_pe``, ``radial_range_m``.
    Raises ``ValueError`` where the reference raises (``transport.py:1072-1073``,
    ``1115-1123``).
    """
    omega = np.asarray(config["omega_per_ns"], float)
    positions = np.asarray(detector["positions_m"], float)
    source = np.asarray(flash["position_m"], float)
    photons = float(flash["photons"])
    t_source = float(flash.get("time_ns", 0.0))
    displacement = positions - source[None, :]
    radii = np.linalg.norm(displacement, axis=1)
    if np.any(radii == 0):
        raise ValueError("isotropic point source cannot coincide with an OM centre")
    toward = source[None, :] - positions
    toward /= np.linalg.norm(toward, axis=1)[:, None]
    cosines = np.sum(np.asarray(detector["orientations"], float) * toward, axis=1)
    area = np.asarray(detector["area_m2"], float)
    efficiency = float(detector["spectral_weight"])
    alpha_full = np.asarray(detector["alpha"], float)
    acceptance = detector.get("acceptance")
    low, high = map(float, config["radial_range_m"])
    inside = (radii >= low) & (radii <= high)
    mu_a = float(table["absorption_per_m"])
    mu_t = mu_a + float(table["scattering_per_m"])
    speed = C_VACUUM_M_PER_NS / float(table["group_index"])
    scale = photons * area * efficiency
    spectrum = np.zeros((len(omega), len(positions), 3), complex)
    # acceptance_spectrum (cache.py:372-436): weights alpha_l P_l(cos) / (4 pi)
    degree = int(table["degree"])
    used = np.zeros(degree + 1)
    used[:min(len(alpha_full), degree + 1)] = alpha_full[:degree + 1]
    significant = np.flatnonzero(np.abs(used) > 1e-12 * np.max(np.abs(used)))
    top = int(significant[-1]) if len(significant) else 0
    acc = (np.asarray(acceptance(cosines), float) if acceptance is not None
           else acceptance_from_alpha(used, cosines))
    if np.any(inside):
        ell = np.arange(top + 1)
        weights = (eval_legendre(ell[None, :], cosines[inside][:, None])
                   * used[None, :top + 1] / (4 * np.pi))
        moments = moments_at(table, radii[inside], top + 1)
        contracted = np.einsum("wrjo,rj->wro", moments, weights)
        value = np.zeros((len(omega), int(inside.sum()), 3), complex)
        value[:, :, 1] = contracted[:, :, 0]
        value[:, :, 2] = contracted[:, :, 1]
        r_in = radii[inside]
        q0_in = np.exp(-mu_t * r_in) / (4 * np.pi * r_in * r_in)
        value[:, :, 0] = (acc[inside] * q0_in)[None, :] * np.exp(
            1j * omega[:, None] * r_in[None, :] / speed)
        spectrum[:, inside] += value * scale[inside][None, :, None]
    q0 = scale * acc * np.exp(-mu_t * radii) / (4 * np.pi * radii * radii)
    outside = ~inside
    if np.any(outside):
        arrival_out = t_source + radii[outside] / speed
        spectrum[:, outside, 0] += q0[outside][None, :] * np.exp(
            1j * omega[:, None] * arrival_out[None, :])
    arrival = t_source + radii / speed
    upper = photons * area * efficiency * acc * np.exp(-mu_a * radii) / (4 * np.pi * radii * radii)
    unsafe = outside & (10 * upper >= float(config["threshold_pe"]))
    if np.any(unsafe):
        raise ValueError(
            f"{int(unsafe.sum())} OMs outside radial_range_m have an absorption-only "
            "estimate above threshold; prepare a cache covering the source-to-OM "
            f"distances (up to {float(np.max(radii[unsafe])):g} m).")
    fastest = float(table["group_index"])
    origins = t_source + radii / (C_VACUUM_M_PER_NS / fastest)
    relative = spectrum * np.exp(-1j * omega[:, None] * origins[None, :])[:, :, None]
    edges = np.asarray(config["edges_ns"], float)
    components = np.zeros((len(positions), len(edges) - 1, 3))
    for order in (1, 2):
        components[:, :, order] = readout_bins(omega, relative[:, :, order], edges,
                                               config.get("readout_omega_per_ns"))
    index = np.searchsorted(edges, arrival - origins, side="right") - 1
    bin_inside = (index >= 0) & (index < len(edges) - 1)
    np.add.at(components[:, :, 0], (np.flatnonzero(bin_inside), index[bin_inside]),
              q0[bin_inside])
    charge = spectrum[0].real
    threshold = float(config["threshold_pe"])
    active = inside & (charge.sum(axis=1) >= threshold)
    if threshold == 0:
        active = inside
    return dict(spectrum_pe=spectrum, components_pe=components, charge_components_pe=charge,
                time_origin_ns=origins, active=active, order0_bin=np.where(bin_inside, index, -1))
