"""Source, detector, configuration and response types of the transport path.

These mirror the reference's public types field for field (``sources.py:81-107``,
``model.py:95-171``, ``transport.py:27-108`` and ``256-383``) so that either
these or the reference's own objects can be passed to the B200 routes: the
routes only read attributes by their reference names.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

import numpy as np

C_VACUUM_M_PER_NS = 0.299792458

__all__ = ["IsotropicFlash", "DetectorArray", "KernelConfig", "TransportResponse",
           "TransportComponent", "acceptance_coefficients", "synthetic_detector",
           "Medium"]


@dataclass(frozen=True)
class IsotropicFlash:
    """Point flash (``sources.py:81-107``): position, photons, wavelength or shape."""
    position_m: np.ndarray
    photons: float
    wavelength_nm: float | None = None
    spectral_shape: Callable[[np.ndarray], np.ndarray] | None = None
    time_ns: float = 0.0

    def __post_init__(self):
        position = np.asarray(self.position_m, float)
        if position.shape != (3,) or not np.isfinite(position).all():
            raise ValueError("position_m must be a finite 3-vector")
        if not np.isfinite(self.photons) or self.photons < 0 or not np.isfinite(self.time_ns):
            raise ValueError("photons must be nonnegative and time_ns finite")
        if (self.wavelength_nm is None) == (self.spectral_shape is None):
            raise ValueError("provide exactly one of wavelength_nm or spectral_shape")
        if self.wavelength_nm is not None and (not np.isfinite(self.wavelength_nm)
                                                or self.wavelength_nm <= 0):
            raise ValueError("wavelength_nm must be positive")
        object.__setattr__(self, "position_m", position)

    @classmethod
    def monochromatic(cls, position_m, photons, wavelength_nm, *, time_ns=0.0):
        return cls(position_m, photons, wavelength_nm=float(wavelength_nm), time_ns=time_ns)

    @classmethod
    def broadband(cls, position_m, photons, spectral_shape, *, time_ns=0.0):
        return cls(position_m, photons, spectral_shape=spectral_shape, time_ns=time_ns)


@dataclass(frozen=True)
class Medium:
    """One band of a homogeneous medium (``medium.py:8-40``)."""
    absorption_per_m: float
    scattering_per_m: float
    g: float
    group_index: float
    wavelength_nm: float = 450.0

    @property
    def extinction_per_m(self):
        return self.absorption_per_m + self.scattering_per_m

    @property
    def speed_m_per_ns(self):
        return C_VACUUM_M_PER_NS / self.group_index


@dataclass(frozen=True)
class DetectorArray:
    """OM array (``model.py:95-171``): geometry plus angular/spectral response."""
    positions_m: np.ndarray
    orientations: np.ndarray
    effective_area_m2: float | np.ndarray
    angular_acceptance: Callable[[np.ndarray], np.ndarray]
    spectral_efficiency: Callable[[np.ndarray], np.ndarray]
    identifiers: dict = field(default_factory=dict)

    def __post_init__(self):
        positions = np.asarray(self.positions_m, float)
        orientations = np.asarray(self.orientations, float)
        if positions.ndim != 2 or positions.shape[1] != 3 or orientations.shape != positions.shape:
            raise ValueError("positions_m and orientations must be (N, 3)")
        orientations = orientations / np.linalg.norm(orientations, axis=1)[:, None]
        object.__setattr__(self, "positions_m", positions)
        object.__setattr__(self, "orientations", orientations)

    def __len__(self):
        return len(self.positions_m)

    def head_on_cosine(self, source_position_m):
        """Cosine +1 when an OM orientation points from OM towards source."""
        toward = np.asarray(source_position_m, float)[None, :] - self.positions_m
        toward /= np.linalg.norm(toward, axis=1)[:, None]
        return np.sum(self.orientations * toward, axis=1)

    def spectral_weight(self, wavelength_nm):
        value = np.asarray(self.spectral_efficiency(np.asarray(wavelength_nm, float)), float)
        if not np.isfinite(value).all() or np.any(value < 0):
            raise ValueError("nonfinite or negative detector spectral response")
        return value


def synthetic_detector(clusters=1):
    """The reference's synthetic Baikal-like array (``examples/synthetic.py:20-54``)."""
    from .workloads import baikal_like_positions
    positions, orientations = baikal_like_positions(clusters=clusters)

    def angular_acceptance(cosine):
        x = np.asarray(cosine, float)
        return .45 + .45 * x + .10 * x * x

    def spectral_efficiency(wavelength_nm):
        wavelength = np.asarray(wavelength_nm, float)
        return .20 * np.exp(-0.5 * ((wavelength - 450.) / 90.) ** 2)

    return DetectorArray(positions, orientations, np.pi * .20 ** 2, angular_acceptance,
                         spectral_efficiency)


def acceptance_coefficients(acceptance, degree, *, quadrature_order=512):
    """``alpha_l = 2 pi int A(x) P_l(x) dx`` by Gauss-Legendre (``cache.py:81-99``)."""
    from numpy.polynomial.legendre import leggauss
    x, w = leggauss(int(quadrature_order))
    values = np.asarray(acceptance(x), dtype=float)
    if values.shape != x.shape or not np.isfinite(values).all():
        raise ValueError("acceptance must map an array of cosines to finite values")
    if np.any(values < 0):
        raise ValueError("acceptance must be nonnegative")
    out = np.zeros(int(degree) + 1)
    p_prev, p = np.ones_like(x), x.copy()
    for ell in range(int(degree) + 1):
        if ell == 0:
            basis = np.ones_like(x)
        elif ell == 1:
            basis = x
        else:
            basis = ((2 * ell - 1) * x * p - (ell - 1) * p_prev) / ell
            p_prev, p = p, basis
        out[ell] = 2 * np.pi * np.sum(basis * w * values)
    return out


@dataclass(frozen=True)
class KernelConfig:
    """The settings of ``KernelConfig`` (``transport.py:27-108``) this path reads."""
    omega_per_ns: np.ndarray = field(default_factory=lambda: np.linspace(0.0, 1.2, 321))
    relative_time_edges_ns: np.ndarray = field(
        default_factory=lambda: np.arange(-60.0, 740.0 + 5.0, 5.0))
    radial_range_m: tuple = (3.0, 300.0)
    threshold_pe: float = 0.01
    readout_omega_per_ns: np.ndarray | None = None
    scattered_receiver: str = "centre"

    def __post_init__(self):
        omega = np.asarray(self.omega_per_ns, float)
        edges = np.asarray(self.relative_time_edges_ns, float)
        if (omega.ndim != 1 or not len(omega) or omega[0] != 0
                or not np.isfinite(omega).all() or np.any(np.diff(omega) <= 0)):
            raise ValueError("omega_per_ns must increase from zero")
        readout = (None if self.readout_omega_per_ns is None
                   else np.asarray(self.readout_omega_per_ns, float))
        if readout is not None and (
                readout.ndim != 1 or len(readout) < 2 or readout[0] != 0
                or not np.isclose(readout[-1], omega[-1], rtol=0, atol=1e-12)
                or not np.isfinite(readout).all() or np.any(np.diff(readout) <= 0)):
            raise ValueError("readout_omega_per_ns must increase from zero to the cache cutoff")
        if (edges.ndim != 1 or len(edges) < 2 or not np.isfinite(edges).all()
                or np.any(np.diff(edges) <= 0)):
            raise ValueError("relative_time_edges_ns must strictly increase")
        if not 0 <= self.threshold_pe or not np.isfinite(self.threshold_pe):
            raise ValueError("threshold_pe must be finite and nonnegative")
        object.__setattr__(self, "omega_per_ns", omega)
        object.__setattr__(self, "readout_omega_per_ns", readout)
        object.__setattr__(self, "relative_time_edges_ns", edges)


@dataclass
class TransportComponent:
    charge_pe: np.ndarray
    bins_pe: np.ndarray
    time_origin_ns: np.ndarray
    relative_time_edges_ns: np.ndarray
    active: np.ndarray


@dataclass
class TransportResponse:
    """Response folded over wavelength and OM efficiency (``transport.py:256-328``).

    ``spectrum_pe`` (frequency, OM, order), ``components_pe`` (OM, bin, order),
    ``charge_components_pe`` (OM, order). Arrays may be NumPy or torch tensors
    (device-resident responses of the batched API).
    """
    detector: object
    omega_per_ns: np.ndarray
    relative_time_edges_ns: np.ndarray
    spectrum_pe: object
    components_pe: object
    charge_components_pe: object
    time_origin_ns: object
    active: object
    method: str
    metadata: dict

    @property
    def charge_pe(self):
        return self.charge_components_pe.sum(axis=1)

    @property
    def bins_pe(self):
        return self.components_pe.sum(axis=2)

    def select(self, component="all"):
        choices = {0: (0,), 1: (1,), 2: (2,), "0": (0,), "1": (1,),
                   ">=2": (2,), "0+1": (0, 1), "all": (0, 1, 2)}
        if component not in choices:
            raise ValueError("component must be 0, 1, >=2, 0+1 or all")
        sel = list(choices[component])
        return TransportComponent(self.charge_components_pe[:, sel].sum(axis=1),
                                  self.components_pe[:, :, sel].sum(axis=2),
                                  self.time_origin_ns, self.relative_time_edges_ns, self.active)
