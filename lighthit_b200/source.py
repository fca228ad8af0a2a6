"""Order >=2 source compile on the B200: the axial-slice basis of a shower.

Reference: ``node_sources`` (``shower/ge2.py:35-67``) compiling each node band
of the band fold with ``compile_axial_slices`` (``_shower_basis.py:188-645``)
and the shower basis (``ShowerBasis``: 0.25 m slices, cubic axial weights,
5-moment stencil of 0.2 m for slices wider than 0.03 m, 0.02 ns linear time
lattice). The lattice sizes and the frame are small host computations; the
deposit, time-lattice transform and stencil run in ``liblh_b200.so``.
"""
from __future__ import annotations

import ctypes as C
import functools
from dataclasses import dataclass

import numpy as np

from . import _lib

__all__ = ["ShowerBasisSettings", "SourceCompiler", "axis_frame", "harmonic_layout"]


@dataclass(frozen=True)
class ShowerBasisSettings:
    """The ``ShowerBasis`` fields the compile reads (``shower_basis.py:61-76``)."""
    cell_m: float = 0.25
    stencil_m: float = 0.2
    stencil_threshold_m: float = 0.03
    time_step_ns: float = 0.02


def harmonic_layout(degree, max_m):
    """``(starts, aa, bb, kept, channel_degree)`` of ``axial_fast._layout``."""
    starts, kept, ell_of = [0], [], []
    for ell in range(degree + 1):
        for m in range(-min(ell, max_m), min(ell, max_m) + 1):
            kept.append(ell * ell + ell + m)
            ell_of.append(ell)
        starts.append(len(kept))
    aa = np.zeros((degree + 1, max_m + 1))
    bb = aa.copy()
    for m in range(max_m + 1):
        for ell in range(m + 2, degree + 1):
            aa[ell, m] = np.sqrt((4 * ell * ell - 1) / (ell * ell - m * m))
            bb[ell, m] = np.sqrt(((2 * ell + 1) * ((ell - 1) ** 2 - m * m))
                                 / ((2 * ell - 3) * (ell * ell - m * m)))
    return (np.asarray(starts, np.int64), aa, bb, np.asarray(kept, np.int64),
            np.asarray(ell_of, np.int64))


def axis_frame(start, direction, length, weights):
    """``AxisFrame.of`` (``axial_source.py:88-118``): centre, axis, first, second."""
    start = np.ascontiguousarray(start, float)
    direction = np.ascontiguousarray(direction, float)
    length = np.ascontiguousarray(length, float)
    share = np.ascontiguousarray(np.asarray(weights, float) / np.sum(weights))
    # Bit for bit the reference's frame (one rounding apart can move a node
    # across a slice edge or a slice across the stencil threshold): its centre
    # expression and its einsum("i,ij,ik->jk") covariance, which add the
    # elements in order, summed in one host pass of the library (the lower
    # triangle: eigh reads only that).
    centre = np.zeros(3)
    covariance = np.zeros((3, 3))
    _lib.check(_lib.load().lh_axis_frame_sums(
        len(length), start.ctypes.data, direction.ctypes.data, length.ctypes.data,
        share.ctypes.data, centre.ctypes.data, covariance.ctypes.data), "lh_axis_frame_sums")
    values, vectors = np.linalg.eigh(covariance)
    if np.max(np.abs(values)) <= 1e-24:
        axis = np.sum(share[:, None] * direction, axis=0)
        if np.linalg.norm(axis) <= 1e-12:
            _, angular = np.linalg.eigh(np.einsum("i,ij,ik->jk", share, direction, direction))
            axis = angular[:, -1]
    else:
        axis = vectors[:, int(np.argmax(values))]
    axis = axis / np.linalg.norm(axis)
    if float((share * (direction @ axis)).sum()) < 0:
        axis = -axis
    helper = np.array([0.0, 0.0, 1.0])
    if abs(float(axis @ helper)) > 0.9:
        helper = np.array([1.0, 0.0, 0.0])
    first = _cross(axis, helper)
    first /= np.linalg.norm(first)
    return centre, axis, first, _cross(axis, first)


@functools.lru_cache(maxsize=8)
def _gauss_rule(order):
    x, w = np.polynomial.legendre.leggauss(order)
    x.flags.writeable = False
    w.flags.writeable = False
    return x, w


def _gauss_legendre(order):
    """Gauss-Legendre nodes and weights (``leggauss``, which solves an eigenvalue
    problem on every call), computed once per order."""
    return _gauss_rule(int(order))


def _cross(a, b):
    """``np.cross`` of two 3-vectors (the same products and differences, without
    its axis bookkeeping, which costs more than the arithmetic here)."""
    a0, a1, a2 = float(a[0]), float(a[1]), float(a[2])
    b0, b1, b2 = float(b[0]), float(b[1]), float(b[2])
    return np.array([a1 * b2 - a2 * b1, a2 * b0 - a0 * b2, a0 * b1 - a1 * b0])


class SourceCompiler:
    """Node bands (wavelength, phase index, fold scale) and layout on the device."""

    def __init__(self, wavelengths_nm, phase_index, scale, degree, azimuthal_degree, omega, *,
                 settings=ShowerBasisSettings(), device="cuda"):
        import torch
        self.device = torch.device(device)
        self.wavelengths = np.asarray(wavelengths_nm, float)
        self.phase = np.asarray(phase_index, float)
        self.scale = np.asarray(scale, float)
        if not (len(self.wavelengths) == len(self.phase) == len(self.scale) <= 8):
            raise ValueError("one wavelength, phase index and scale per node band (<= 8)")
        self.degree, self.azimuthal_degree = int(degree), int(azimuthal_degree)
        self.max_m = min(self.degree, self.azimuthal_degree)
        self.starts, self.aa, self.bb, self.kept, self.channel_degree = harmonic_layout(
            self.degree, self.max_m)
        self.nch = len(self.kept)
        self.settings = settings
        self.omega = np.asarray(omega, float)
        self._omega = torch.tensor(self.omega, dtype=torch.float64, device=self.device)
        self._workspace = None

    def _template(self):
        """The event-independent fields (bands, harmonic layout, basis settings)."""
        if getattr(self, "_fixed", None) is not None:
            return self._fixed
        p = _lib.SourceProblem()
        nb = len(self.wavelengths)
        p.n_bands = nb
        s0 = 1.0 / self.wavelengths ** 2
        s2 = s0 / self.phase ** 2
        for k in range(nb):
            p.band_s0[k], p.band_s2[k] = float(s0[k]), float(s2[k])
            p.band_phase[k], p.band_scale[k] = float(self.phase[k]), float(self.scale[k])
        p.degree, p.max_m, p.nch = self.degree, self.max_m, self.nch
        for k, v in enumerate(self.starts):
            p.starts[k] = int(v)
        for k, v in enumerate(self.channel_degree):
            p.channel_degree[k] = int(v)
        for k, (a, b) in enumerate(zip(self.aa.ravel(), self.bb.ravel())):
            p.aa[k], p.bb[k] = float(a), float(b)
        s = self.settings
        p.cell_m, p.stencil_m = s.cell_m, s.stencil_m
        p.stencil_threshold_m, p.time_step_ns = s.stencil_threshold_m, s.time_step_ns
        p.n_omega = len(self.omega)
        p.omega = self._omega.data_ptr()
        self._fixed = p
        return p

    def problem(self, arrays, frame, n_el, order, fractions, weights, reference, z_origin,
                n_slices, kmax):
        p = _lib.SourceProblem.from_buffer_copy(self._template())
        p.n_el = n_el
        for name in ("start", "direction", "length", "c0", "c2", "beta", "t0", "t1"):
            setattr(p, name, arrays[name].data_ptr())
        centre, axis, first, second = frame
        for k in range(3):
            p.centre[k], p.first[k], p.second[k], p.axis[k] = centre[k], first[k], second[k], axis[k]
        p.element_order = order
        for k in range(order):
            p.node_fraction[k], p.node_weight[k] = float(fractions[k]), float(weights[k])
        p.reference_ns, p.z_origin = reference, z_origin
        p.n_slices, p.kmax = n_slices, kmax
        return p

    def band(self, b):
        """This compiler restricted to node band ``b`` (its own workspace)."""
        view = SourceCompiler.__new__(SourceCompiler)
        view.__dict__.update(self.__dict__)
        view.wavelengths, view.phase = self.wavelengths[b:b + 1], self.phase[b:b + 1]
        view.scale = self.scale[b:b + 1]
        view._workspace, view._fixed = None, None
        return view

    def compile(self, elements, frame=None, *, stream=None, check=True, status=None,
                device_elements=None):
        """Points and channels of every node band (device), the emission reference.

        ``elements``: reference ``SpectralLightElements`` or a dict with its
        field names. Returns ``(points (band, P, 3) [z, x, y], channels (band, P,
        nch, W) complex64, n_points (band,), reference_ns, frame)``. When every
        element is above the Cherenkov threshold in every node band, all bands
        share one lattice and ``reference_ns`` is a float; otherwise each band
        compiles its own emitting elements (``_band_field``, ``shower/ge2.py:21-32``)
        on its own lattice, a band without them takes another band's points with
        zero channels (``node_sources``, ``:35-67``), and ``reference_ns`` is an
        array of one emission reference per band.
        """
        import torch

        def field(name):
            return np.asarray(elements[name] if isinstance(elements, dict)
                              else getattr(elements, name), float)

        start, direction, length = field("start_m"), field("direction"), field("length_m")
        c0, c2, beta = field("coefficient0"), field("coefficient2"), field("beta")
        t0, t1 = field("start_ns"), field("end_ns")
        # rounding is monotone: beta n <= 1 for some band iff it holds at the smallest n
        if np.any(beta * float(np.min(self.phase)) <= 1):
            return self._compile_per_band(elements, beta, frame, stream=stream, check=check,
                                          status=status)
        if frame is None:
            frame = axis_frame(start, direction, length, c0)
        centre, axis = np.asarray(frame[0], float), np.asarray(frame[1], float)
        s = self.settings
        order = 1 if float(np.max(length)) <= s.cell_m / 10 else 2
        x, w = _gauss_legendre(order)
        fractions, weights = (x + 1) / 2, w / 2
        reference = float(t0.min())
        # axial coordinates as start.axis + f length (direction.axis): matrix-vector
        # products instead of (N, 3) temporaries (the lattice sizes only)
        z_start = start @ axis - float(centre @ axis)
        z_step = length * (direction @ axis)
        z_mid = z_start + 0.5 * z_step
        z_origin = float(z_mid.min()) - 2 * s.cell_m
        z_nodes = np.concatenate([z_start + f * z_step for f in fractions])
        t_nodes = np.concatenate([t0 + f * (t1 - t0) for f in fractions])
        kmax = int(np.floor((float(t_nodes.max()) - reference) / s.time_step_ns)) + 3
        zb = np.floor((z_nodes - z_origin) / s.cell_m)
        if zb.min() < 1:
            raise NotImplementedError("chord nodes reach below the slice lattice origin")
        n_slices = int(zb.max()) + 3
        dev = self.device
        if device_elements is None:
            arrays = {k: _lib.upload(v, torch.float64, dev)
                      for k, v in dict(start=start, direction=direction, length=length, c0=c0,
                                       c2=c2, beta=beta, t0=t0, t1=t1).items()}
        else:
            d = device_elements
            arrays = dict(start=d["start_m"], direction=d["direction"], length=d["length_m"],
                          c0=d["coefficient0"], c2=d["coefficient2"], beta=d["beta"],
                          t0=d["start_ns"], t1=d["end_ns"])
        p = self.problem(arrays, frame, len(length), order, fractions, weights, reference,
                         z_origin, n_slices, kmax)
        nb = len(self.wavelengths)
        capacity = 5 * n_slices
        points = torch.empty((nb, capacity, 3), dtype=torch.float64, device=dev)
        channels = torch.empty((nb, capacity, self.nch, len(self.omega)), dtype=torch.complex64,
                               device=dev)
        n_points = torch.zeros(nb, dtype=torch.int32, device=dev)
        out = _lib.SourceOutput(capacity, points.data_ptr(), channels.data_ptr(),
                                n_points.data_ptr())
        lib = _lib.load()
        need = int(lib.lh_source_workspace_bytes(C.byref(p)))
        if need == 0:
            raise ValueError("source compile problem rejected by the device library")
        if self._workspace is None or self._workspace.numel() < need:
            self._workspace = torch.empty(need, dtype=torch.uint8, device=dev)
        own_status = status is None
        if own_status:
            status = torch.zeros(1, dtype=torch.int32, device=dev)
        sp = _lib.stream_ptr(stream or torch.cuda.current_stream(dev))
        _lib.check(lib.lh_source_compile(C.byref(p), C.byref(out), self._workspace.data_ptr(),
                                         self._workspace.numel(), status.data_ptr(), sp),
                   "lh_source_compile")
        self._keep = arrays
        if own_status and check and int(status.item()) & _lib.LH_STATUS_OVERFLOW:
            raise ValueError("element nodes fall outside the source lattice")
        return points, channels, n_points, reference, frame

    def _compile_per_band(self, elements, beta, frame, *, stream, check, status):
        """``node_sources`` for elements above threshold in only some node bands:
        one compile per band on its emitting elements, padded to one layout."""
        import torch
        names = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
                 "start_ns", "end_ns")
        el = {k: np.asarray(elements[k] if isinstance(elements, dict) else getattr(elements, k),
                            float) for k in names}
        if frame is None:
            frame = axis_frame(el["start_m"], el["direction"], el["length_m"],
                               el["coefficient0"])
        if not hasattr(self, "_bands"):
            self._bands = [self.band(b) for b in range(len(self.phase))]
        parts = {}
        for b, phase in enumerate(self.phase):
            mask = beta * float(phase) > 1
            if np.any(mask):
                sub = {k: v[mask] for k, v in el.items()}
                parts[b] = self._bands[b].compile(sub, frame, stream=stream, check=check,
                                                  status=status)
        if not parts:
            raise ValueError("no element emits in any node band")
        nb = len(self.phase)
        template = parts[min(parts)]
        capacity = max(int(p[0].shape[1]) for p in parts.values())
        dev = self.device
        points = torch.zeros((nb, capacity, 3), dtype=torch.float64, device=dev)
        channels = torch.zeros((nb, capacity, self.nch, len(self.omega)), dtype=torch.complex64,
                               device=dev)
        n_points = torch.zeros(nb, dtype=torch.int32, device=dev)
        reference = np.zeros(nb)
        for b in range(nb):
            pts, ch, npts, ref, _ = parts.get(b, template)
            cap = int(pts.shape[1])
            points[b, :cap] = pts[0]
            if b in parts:
                channels[b, :cap] = ch[0]
            n_points[b] = npts[0]
            reference[b] = ref
        return points, channels, n_points, reference, frame
