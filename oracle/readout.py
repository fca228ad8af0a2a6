"""Oracle: spectrum -> time bins (reference ``readout.py``).

SciPy's ``CubicSpline`` (default not-a-knot boundary; scipy 1.18.1 here, the
reference pins ``scipy>=1.11`` in ``pyproject.toml:13``) is the reference's own
interpolant for the 65 -> 321 frequency refinement, so the oracle calls it
directly.
"""
import numpy as np
from scipy.interpolate import CubicSpline


def frequency_weights(omega):
    """Trapezoid weights of a half-axis frequency grid (``readout.py:9-15``)."""
    omega = np.asarray(omega, float)
    step = np.diff(omega)
    return np.r_[step[0] / 2, (step[:-1] + step[1:]) / 2, step[-1] / 2]


def inverse_bins(omega, spectrum, edges_ns):
    """Half-axis Fourier integral, exact per bin (``readout.py:18-40``, sigma 0).

    ``spectrum`` is (frequency, observation); the result is (observation, bin).
    """
    omega = np.asarray(omega, float)
    edges = np.asarray(edges_ns, float)
    w = frequency_weights(omega)
    width = np.diff(edges)
    center = (edges[:-1] + edges[1:]) / 2
    kernel = (width[:, None] * np.sinc(width[:, None] * omega / (2 * np.pi))
              * np.exp(-1j * center[:, None] * omega) * (w / np.pi))
    return (kernel @ np.asarray(spectrum, complex)).real.T


def readout_bins(omega, spectrum, edges_ns, readout_omega=None):
    """``readout.py:43-72``: optional cubic refinement, then ``inverse_bins``."""
    omega = np.asarray(omega, float)
    spectrum = np.asarray(spectrum, complex)
    grid = omega
    if readout_omega is not None and len(omega) > 1:
        readout = np.asarray(readout_omega, float)
        same = len(readout) == len(omega) and np.allclose(readout, omega)
        if not same and np.isclose(readout[-1], omega[-1], rtol=0, atol=1e-12):
            spectrum = (CubicSpline(omega, spectrum.real, axis=0)(readout)
                        + 1j * CubicSpline(omega, spectrum.imag, axis=0)(readout))
            grid = readout
    return inverse_bins(grid, spectrum, edges_ns)
