"""Oracle: order >=2 contraction of axial-basis sources with band-folded kernels.

Restates ``apply_folded`` (``shower/ge2.py:99-119``) ->
``apply_multi_spectral`` (``_shower_basis.py:1126-1198``) ->
``_apply_multi_spectral`` (``_shower_basis.py:894-1050``) with the Wigner
small-d recurrence and real harmonics of ``_directional_numba.py:37-128,389-397``
in float64 NumPy (loops over OM and point, vectorised over band and frequency).
"""
import ctypes as C
from math import exp, lgamma

import numpy as np

from .build import build

_LIB = None


def _apply_c(points, receivers, looks, channels, out_scale, starts, degree, max_m, max_out, alpha,
             pair_lambda, pair_mu, log_r, coefficients, absorption, velocity, omega, flight,
             radial_low, radial_high):
    """``apply_multi_spectral_local`` in C (``o2c_apply``): (receiver, frequency)."""
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(str(build()))
        _LIB.o2c_apply.restype = C.c_int

    def f(a):
        return np.ascontiguousarray(a, dtype=np.float64)

    def c(a):
        return np.ascontiguousarray(a, dtype=np.complex128)

    def i(a):
        return np.ascontiguousarray(a, dtype=np.int64)

    def p(a):
        return C.c_void_p(a.ctypes.data)

    points, receivers, looks = f(points), f(receivers), f(looks)
    channels, coefficients = c(channels), c(coefficients)
    out_scale, alpha, log_r = f(out_scale), f(alpha), f(log_r)
    absorption, velocity, omega = f(absorption), f(velocity), f(omega)
    starts, pair_lambda, pair_mu = i(starts), i(pair_lambda), i(pair_mu)
    result = np.zeros((len(receivers), len(omega)), complex)
    rc = _LIB.o2c_apply(C.c_int64(len(points)), p(points), C.c_int64(len(receivers)), p(receivers),
                        p(looks), C.c_int(channels.shape[0]), C.c_int(channels.shape[2]),
                        p(channels), p(out_scale), p(starts), C.c_int(degree), C.c_int(max_m),
                        C.c_int(max_out), p(alpha), C.c_int(len(pair_lambda)), p(pair_lambda),
                        p(pair_mu), C.c_int(len(log_r)), p(log_r), p(coefficients),
                        p(absorption), p(velocity), C.c_int(len(omega)), p(omega),
                        C.c_int(int(bool(flight))), C.c_double(radial_low),
                        C.c_double(radial_high), p(result))
    if rc:
        raise MemoryError("oracle order >=2 apply: scratch allocation failed")
    return result


def parity(n):
    return 1.0 if n % 2 == 0 else -1.0


def start_norm_table(jmax):
    """``sqrt(binom(2j, j - nu))`` (``_directional_numba.py:389-397``)."""
    table = np.zeros((jmax + 1, 2 * jmax + 1))
    for j in range(jmax + 1):
        for nu in range(-j, j + 1):
            table[j, nu + jmax] = exp(0.5 * (lgamma(2 * j + 1) - lgamma(j + nu + 1)
                                             - lgamma(j - nu + 1)))
    return table


def start_value(j, mu, nu, half_cos, half_sin, start_norm, jmax):
    """``d^j_(mu nu)`` at ``j = max(|mu|, |nu|)`` (``_directional_numba.py:37-48``)."""
    sign = 1.0
    if abs(nu) == j and abs(mu) != j:
        mu, nu = nu, mu
        sign *= parity(mu - nu)
    if mu == -j:
        mu = j
        nu = -nu
        sign *= parity(j + nu)
    return sign * start_norm[j, nu + jmax] * half_cos ** (j + nu) * (-half_sin) ** (j - nu)


def wigner(degree, max_out, max_in, cosine, start_norm, jmax):
    """``out[l, nu + max_out, mu] = d^l_(mu nu)`` for mu in 0..max_in (``:51-87``)."""
    out = np.zeros((degree + 1, 2 * max_out + 1, max_in + 1))
    half_cos = np.sqrt((1.0 + cosine) / 2.0)
    half_sin = np.sqrt((1.0 - cosine) / 2.0)
    for nu in range(-max_out, max_out + 1):
        for mu in range(max_in + 1):
            start = max(abs(nu), mu)
            if start > degree:
                continue
            previous = 0.0
            current = start_value(start, mu, nu, half_cos, half_sin, start_norm, jmax)
            out[start, nu + max_out, mu] = current
            for ell in range(start, degree):
                if ell == 0:
                    value = cosine * current
                else:
                    lower = (ell * ell - mu * mu) * (ell * ell - nu * nu)
                    lower = np.sqrt(lower) if lower > 0.0 else 0.0
                    upper = np.sqrt(((ell + 1) ** 2 - mu * mu) * ((ell + 1) ** 2 - nu * nu))
                    value = (((2 * ell + 1) * (ell * (ell + 1) * cosine - mu * nu) * current
                              - (ell + 1) * lower * previous) / (ell * upper))
                previous = current
                current = value
                out[ell + 1, nu + max_out, mu] = current
    return out


def harmonics(x, y, z, degree):
    """Real orthonormal harmonics, flat ``l*l+l+m`` (``_directional_numba.py:90-128``)."""
    out = np.zeros((degree + 1) ** 2)
    radius = np.sqrt(x * x + y * y + z * z)
    mu = z / radius
    transverse = np.sqrt(x * x + y * y)
    sine = transverse / radius
    cp = 1.0 if transverse == 0.0 else x / transverse
    sp = 0.0 if transverse == 0.0 else y / transverse
    cm, sm = 1.0, 0.0
    diagonal = 1.0 / np.sqrt(4 * np.pi)
    v0 = v1 = 0.0
    for m in range(degree + 1):
        if m:
            diagonal *= np.sqrt((2.0 * m + 1) / (2.0 * m)) * sine
            cm, sm = cm * cp - sm * sp, sm * cp + cm * sp
        v0 = diagonal
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
                out[centre] = value
            else:
                out[centre - m] = np.sqrt(2) * value * sm
                out[centre + m] = np.sqrt(2) * value * cm
    return out


def erow_table(ell, wig, cosines, sines, max_out, max_m):
    """Real rotation row block for degree ``ell`` (``_shower_basis.py:957-977``)."""
    root2 = np.sqrt(2.0)
    erow = np.zeros((2 * max_out + 1, 2 * max_m + 1))
    erow[max_out, max_m] = wig[ell, max_out, 0]
    top_n = min(ell, max_m)
    top_p = min(ell, max_out)
    for n in range(1, top_n + 1):
        base = root2 * parity(n) * wig[ell, max_out, n]
        erow[max_out, max_m + n] = base * cosines[n]
        erow[max_out, max_m - n] = base * sines[n]
    for p in range(1, top_p + 1):
        erow[max_out + p, max_m] = root2 * parity(p) * wig[ell, max_out + p, 0]
        for n in range(1, top_n + 1):
            cross = parity(p) * wig[ell, max_out + p, n]
            straight = wig[ell, max_out - p, n]
            cc = parity(n) * (cross + straight)
            ss = parity(n) * (cross - straight)
            erow[max_out + p, max_m + n] = cc * cosines[n]
            erow[max_out + p, max_m - n] = cc * sines[n]
            erow[max_out - p, max_m + n] = -ss * sines[n]
            erow[max_out - p, max_m - n] = ss * cosines[n]
    return erow


def apply_multi_spectral_local(points, receivers, looks, channels, out_scale, starts, degree,
                               max_m, max_out, alpha, pair_lambda, pair_mu, log_r, coefficients,
                               absorption, velocity, omega, flight, radial_low, radial_high):
    """``_apply_multi_spectral`` (``_shower_basis.py:894-1050``), no tolerance screen.

    ``channels`` (band, point, channel, frequency); ``coefficients`` (band,
    interval, degree, pair, power, frequency). Returns (receiver, frequency).
    """
    nlam = coefficients.shape[0]
    width = 2 * max_out + 1
    jmax = max(max_m, max_out)
    start_norm = start_norm_table(jmax)
    result = np.zeros((len(receivers), len(omega)), complex)
    for index in range(len(receivers)):
        for cell in range(len(points)):
            dx, dy, dz = receivers[index] - points[cell]
            radius = np.sqrt(dx * dx + dy * dy + dz * dz)
            if radius < radial_low or radius > radial_high:
                continue
            cosine = min(max(dz / radius, -1.0), 1.0)
            phi = np.arctan2(dy, dx)
            transverse = np.sqrt(dx * dx + dy * dy)
            sine = transverse / radius
            cp = 1.0 if transverse == 0.0 else dx / transverse
            sp = 0.0 if transverse == 0.0 else dy / transverse
            cosines = np.cos(np.arange(max_m + 1) * phi)
            sines = np.sin(np.arange(max_m + 1) * phi)
            lx, ly, lz = looks[index]
            a1 = cosine * cp * lx + cosine * sp * ly - sine * lz
            a2 = -sp * lx + cp * ly
            a3 = sine * cp * lx + sine * sp * ly + cosine * lz
            detector = harmonics(a1, a2, a3, max_out)
            wig = wigner(degree, max_out, max_m, cosine, start_norm, jmax)
            logr = np.log(radius)
            j = int(np.clip(np.searchsorted(log_r, logr, side="right") - 1, 0, len(log_r) - 2))
            t = logr - log_r[j]
            scale = out_scale[:, index] * np.exp(-absorption * radius) / (4 * np.pi * radius * radius)
            if flight:
                scale_phase = scale[:, None] * np.exp(1j * omega[None, :] * radius / velocity[:, None])
            else:
                scale_phase = scale[:, None] * np.ones(len(omega))
            response = np.zeros((nlam, len(omega)), complex)
            for ell in range(degree + 1):
                erow = erow_table(ell, wig, cosines, sines, max_out, max_m)
                keep = min(ell, max_m)
                centre = starts[ell] + keep
                top_p = min(ell, max_out)
                cols = [centre + (b - max_m) for b in range(max_m - keep, max_m + keep + 1)]
                block = channels[:, cell, cols, :]  # (lam, b, w)
                rotated = np.einsum("ab,lbw->law", erow[:, max_m - keep:max_m + keep + 1], block)
                cubic = coefficients[:, j, ell]  # (lam, pair, power, w)
                radial = ((cubic[:, :, 0] * t + cubic[:, :, 1]) * t + cubic[:, :, 2]) * t + cubic[:, :, 3]
                channel_sum = np.zeros((nlam, width, len(omega)), complex)
                for p in range(len(pair_lambda)):
                    lam_d, mu_p = int(pair_lambda[p]), int(pair_mu[p])
                    if mu_p > top_p:
                        continue
                    dc = lam_d * lam_d + lam_d
                    positive = alpha[lam_d] * detector[dc + mu_p]
                    negative = alpha[lam_d] * detector[dc - mu_p] if mu_p else 0.0
                    if negative != 0.0:
                        channel_sum[:, max_out - mu_p] += negative * radial[:, p]
                    if positive != 0.0:
                        channel_sum[:, max_out + mu_p] += positive * radial[:, p]
                sel = slice(max_out - top_p, max_out + top_p + 1)
                response += np.sum(rotated[:, sel] * channel_sum[:, sel], axis=1)
            result[index] += np.sum(response * scale_phase, axis=0)
    return result


def apply_folded(folded, sources, positions, looks, alpha, area, window, *, fast=False):
    """``apply_folded`` -> ``apply_multi_spectral`` for sources sharing one point set
    (``fast``: the same loops in C, ``oracle/ge2.c``).

    ``sources``: dict with ``points_m`` (P,3), ``channels`` (band, P, nch, W),
    ``reference_ns`` (band,), ``frame`` (centre, first, second, axis),
    ``degree``, ``azimuthal_degree``. Returns (frequency, OM).
    """
    omega = np.asarray(folded["omega"], float)
    frame = sources["frame"]
    centre = np.asarray(frame["centre"], float)
    basis = np.stack([frame["first"], frame["second"], frame["axis"]])

    def rotate(v):
        return np.asarray(v, float) @ basis.T

    ref = np.asarray(sources["reference_ns"], float)
    reference = float(ref.min())
    channels = np.asarray(sources["channels"], complex) * np.exp(
        1j * omega[None, :] * (ref - reference)[:, None])[:, None, None, :]
    degree = int(sources["degree"])
    az = int(sources["azimuthal_degree"])
    starts = [0]
    for ell in range(degree + 1):
        starts.append(starts[-1] + 2 * min(ell, az) + 1)
    low, high = map(float, window)
    max_m = min(az, int(folded["degree"]))
    acc = int(folded["acceptance_degree"])
    out_scale = np.repeat(np.asarray(area, float)[None, :], channels.shape[0], axis=0)
    if fast:
        result = _apply_c(
            rotate(np.asarray(sources["points_m"], float) - centre),
            rotate(np.asarray(positions) - centre), rotate(looks), channels, out_scale,
            np.asarray(starts), int(folded["degree"]), max_m, acc, np.asarray(alpha, float)[:acc + 1],
            folded["pair_lambda"], folded["pair_mu"], np.asarray(folded["log_r"], float),
            np.asarray(folded["coefficients"]), np.asarray(folded["absorption"], float),
            np.asarray(folded["speed"], float), omega, str(folded["phase"]) == "flight", low, high)
        return result.T * np.exp(1j * omega * reference)[:, None]
    result = apply_multi_spectral_local(
        rotate(np.asarray(sources["points_m"], float) - centre), rotate(np.asarray(positions) - centre),
        rotate(looks), channels, out_scale, np.asarray(starts), int(folded["degree"]), max_m, acc,
        np.asarray(alpha, float)[:acc + 1], folded["pair_lambda"], folded["pair_mu"],
        np.asarray(folded["log_r"], float), np.asarray(folded["coefficients"]),
        np.asarray(folded["absorption"], float), np.asarray(folded["speed"], float), omega,
        str(folded["phase"]) == "flight", low, high)
    return result.T * np.exp(1j * omega * reference)[:, None]
