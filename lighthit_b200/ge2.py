"""Order >=2 on the B200: ``apply_folded`` for node-band axial sources.

Reference: ``apply_folded`` (``shower/ge2.py:99-119``) ->
``apply_multi_spectral`` (``_shower_basis.py:1126-1198``) ->
``_apply_multi_spectral`` (``_shower_basis.py:894-1050``).

The band-folded kernels (``ShowerTransport.tables()['folded']``,
``band_fold.py:155-208``) are built once by the reference and uploaded
read-only as complex64 ``[band][interval][l][pair][power][omega]``. Per call
the host only rotates the points and OMs into the source's axis frame
(float64, O(points + OMs)); the phase alignment of the band sources, the
geometry (float64) and the contraction run in ``liblh_b200.so``: float32 on
the CUDA cores (``mode="fp32"``, and every zero-frequency apply), or on the
tensor cores with BF16 operands and float32 accumulation (``"split-bf16"``:
hi + mid + lo parts, six products, float32 accuracy; ``"bf16"``: one
product), for which the folded kernels are packed once into the tcgen05
operand layout.
"""
from __future__ import annotations

from dataclasses import dataclass
import ctypes as C
from math import exp, lgamma

import numpy as np

from . import _lib

__all__ = ["Ge2Table", "AxialSources", "apply_folded"]


def _start_norm(jmax):
    """``sqrt(binom(2j, j - nu))`` (``_directional_numba.py:389-397``)."""
    table = np.zeros((jmax + 1, 2 * jmax + 1))
    for j in range(jmax + 1):
        for nu in range(-j, j + 1):
            table[j, nu + jmax] = exp(0.5 * (lgamma(2 * j + 1) - lgamma(j + nu + 1)
                                             - lgamma(j - nu + 1)))
    return table


@dataclass
class AxialSources:
    """Node-band sources on one point set (the reference's ``AxialSource`` list).

    ``points_m`` (P, 3) detector coordinates; ``channels`` (band, P, nch, W)
    complex; ``reference_ns`` per band; ``frame`` = (centre, first, second, axis).
    """
    points_m: np.ndarray
    channels: object
    reference_ns: np.ndarray
    frame: tuple
    degree: int
    azimuthal_degree: int

    @classmethod
    def from_reference(cls, sources):
        """From a list of reference ``AxialSource`` objects sharing their points."""
        first = sources[0]
        f = first.frame
        return cls(np.asarray(first.points_m(), float),
                   np.stack([np.asarray(s.channels, np.complex64) for s in sources]),
                   np.array([float(s.reference_ns) for s in sources]),
                   (np.asarray(f.centre_m, float), np.asarray(f.first, float),
                    np.asarray(f.second, float), np.asarray(f.axis, float)),
                   int(first.degree), int(first.azimuthal_degree))


class Ge2Table:
    """Band-folded order >=2 kernels resident on the device."""

    def __init__(self, folded, alpha, *, device="cuda", source_degree=None,
                 azimuthal_degree=None):
        import torch
        self.device = torch.device(device)
        dev = self.device
        coef = np.asarray(folded["coefficients"])
        self.n_bands, self.n_intervals = coef.shape[0], coef.shape[1]
        self.degree = int(folded["degree"])
        self.acc_degree = int(folded["acceptance_degree"])
        self.omega = np.asarray(folded["omega"], float)
        self.pair_lambda = np.asarray(folded["pair_lambda"], np.int32)
        self.pair_mu = np.asarray(folded["pair_mu"], np.int32)
        self.log_r = np.asarray(folded["log_r"], float)
        self.flight = str(folded["phase"]) == "flight"
        self.absorption = np.asarray(folded["absorption"], float)
        self.speed = np.asarray(folded["speed"], float)
        self.alpha = np.ascontiguousarray(np.asarray(alpha, float)[:self.acc_degree + 1])
        sd = self.degree if source_degree is None else int(source_degree)
        az = sd if azimuthal_degree is None else int(azimuthal_degree)
        if sd < self.degree:
            raise ValueError("source degree is insufficient")
        self.source_degree, self.azimuthal_degree = sd, az
        self.max_m = min(az, self.degree)
        starts = [0]
        for ell in range(sd + 1):
            starts.append(starts[-1] + 2 * min(ell, az) + 1)
        self.starts = np.asarray(starts, np.int32)
        self.nch = int(starts[-1])
        self.jmax = max(self.max_m, self.acc_degree)
        self._coef = torch.view_as_real(torch.from_numpy(coef.astype(np.complex64))).contiguous().to(dev)

        def f64(x):
            return torch.tensor(np.ascontiguousarray(x, float), dtype=torch.float64, device=dev)

        def i32(x):
            return torch.tensor(np.ascontiguousarray(x, np.int32), dtype=torch.int32, device=dev)

        self._log_r, self._abs, self._speed = f64(self.log_r), f64(self.absorption), f64(self.speed)
        self._omega, self._alpha = f64(self.omega), f64(self.alpha)
        self._pl, self._pm, self._starts = i32(self.pair_lambda), i32(self.pair_mu), i32(self.starts)
        self._norm = f64(_start_norm(self.jmax))
        self.struct = _lib.Ge2Table(
            self.n_bands, self.n_intervals, self.degree, self.acc_degree, self.max_m,
            len(self.pair_lambda), self.nch, len(self.omega), self._coef.data_ptr(),
            self._log_r.data_ptr(), self._abs.data_ptr(), self._speed.data_ptr(),
            self._omega.data_ptr(), self._pl.data_ptr(), self._pm.data_ptr(),
            self._alpha.data_ptr(), self._starts.data_ptr(), self._norm.data_ptr(), self.jmax,
            int(self.flight))
        self._workspace = None
        self._tc_packed = None

    def tc_packed(self):
        """The folded kernels in the tensor-core operand layout (packed on the
        device once), or None when the table's shape does not fit that path."""
        import torch
        if self._tc_packed is None:
            lib = _lib.load()
            need = int(lib.lh_ge2_tc_pack_bytes(self.struct))
            if need == 0:
                self._tc_packed = False
            else:
                packed = torch.empty(need, dtype=torch.uint8, device=self.device)
                _lib.check(lib.lh_ge2_tc_pack(self.struct, packed.data_ptr(), need,
                                              _lib.stream_ptr(torch.cuda.current_stream(
                                                  self.device))), "lh_ge2_tc_pack")
                self._tc_packed = packed
        return self._tc_packed if self._tc_packed is not False else None

    @classmethod
    def load(cls, path, alpha, **kw):
        return cls(dict(np.load(path)), alpha, **kw)

    def band(self, b):
        """A view of node band ``b`` alone (for bands whose point sets differ),
        made once per band and kept with its own workspace and packed kernels."""
        import copy
        views = self.__dict__.setdefault("_band_views", {})
        if b in views:
            return views[b]
        view = copy.copy(self)
        view._band_views = {}
        per_band = self._coef[0].numel() * self._coef.element_size()
        st = _lib.Ge2Table()
        C.pointer(st)[0] = self.struct
        st.n_bands = 1
        st.coef = self._coef.data_ptr() + b * per_band
        st.absorption = self._abs.data_ptr() + 8 * b
        st.speed = self._speed.data_ptr() + 8 * b
        view.struct = st
        view.n_bands = 1
        view._workspace = None
        view._tc_packed = None
        views[b] = view
        return view

    def radial_limits(self):
        return float(np.exp(self.log_r[0])), float(np.exp(self.log_r[-1]))

    def apply(self, sources: AxialSources, positions, looks, out_scale, window=None, *,
              zero_frequency=False, stream=None):
        """``apply_folded``: (frequency, OM) complex128 spectrum on the host.

        ``out_scale`` (OM,) or (band, OM): the detector scale of every band (the
        route passes the effective area). ``zero_frequency`` evaluates only the
        first frequency (``band_fold.zero_frequency``).
        """
        res = self.apply_device(sources, positions, looks, out_scale, window,
                                zero_frequency=zero_frequency, stream=stream)
        import torch
        torch.cuda.synchronize(self.device)
        return res.cpu().numpy().T

    def _prepare(self, sources, positions, looks, out_scale, window, zero_frequency):
        """Host geometry in the axis frame and the device channels of one problem."""
        import torch
        dev = self.device
        positions = np.atleast_2d(np.asarray(positions, float))
        W = 1 if zero_frequency else len(self.omega)
        if sources.degree < self.degree:
            raise ValueError("source degree is insufficient")
        if (sources.azimuthal_degree != self.azimuthal_degree
                or sources.degree != self.source_degree):
            raise ValueError("source angular layout differs from the table's")
        low_c, high_c = self.radial_limits()
        if window is None:
            low, high = low_c, high_c
        else:
            low, high = map(float, window)
            if (not np.isfinite(low) or not np.isfinite(high) or low < low_c - 1e-9
                    or high > high_c + 1e-9 or low >= high):
                raise ValueError("radial window must lie inside the kernel cache")
        centre, e1, e2, e3 = (np.asarray(v, float) for v in sources.frame)
        basis = np.stack([e1, e2, e3])
        pts = (np.asarray(sources.points_m, float) - centre) @ basis.T
        rec = (positions - centre) @ basis.T
        lk = np.atleast_2d(np.asarray(looks, float)) @ basis.T
        if window is None:
            r = np.linalg.norm(pts[None, :, :] - rec[:, None, :], axis=2)
            if np.any(r < low_c) or np.any(r > high_c):
                raise ValueError("Source/receiver distances outside the cache")
        ref = np.asarray(sources.reference_ns, float)
        reference = float(ref.min())
        ch = sources.channels
        if not isinstance(ch, torch.Tensor):
            ch = torch.from_numpy(np.ascontiguousarray(np.asarray(ch), dtype=np.complex64))
        ch = ch.to(dev, torch.complex64)
        if zero_frequency:
            ch = ch[..., :1]
        if ch.shape[0] != self.n_bands or ch.shape[2] != self.nch or ch.shape[3] < W:
            raise ValueError("source channels do not match the folded kernels")
        shift = ref - reference
        if np.any(shift != 0):  # align every band to the earliest emission reference
            ph = _lib.upload(np.exp(1j * np.outer(shift, self.omega[:ch.shape[3]])),
                             torch.complex64, dev)
            ch = ch * ph[:, None, None, :]
        ch = torch.view_as_real(ch.contiguous()).contiguous()
        scale = np.asarray(out_scale, float)
        if scale.ndim == 1:
            scale = np.repeat(scale[None, :], self.n_bands, axis=0)
        if scale.shape != (self.n_bands, len(positions)):
            raise ValueError("out_scale must hold one value per OM (per band)")
        return dict(pts=pts, rec=rec, lk=lk, scale=scale, ch=ch, W=W, low=low, high=high,
                    reference=reference, n_om=len(positions))

    def _problem(self, q, base, result_ptr):
        """The C problem of a prepared ``q`` whose f64 blocks start at device ``base``."""
        offs, at = {}, base
        for key in ("pts", "rec", "lk", "scale"):
            offs[key] = at
            at += 8 * q[key].size
        return _lib.Ge2Problem(len(q["pts"]), offs["pts"], q["ch"].data_ptr(),
                               int(q["ch"].shape[3]), q["W"], q["n_om"], offs["rec"],
                               offs["lk"], offs["scale"], q["low"], q["high"], q["reference"],
                               result_ptr), at

    def apply_device(self, sources, positions, looks, out_scale, window=None, *,
                     zero_frequency=False, stream=None):
        """One problem: device (OM, frequency) complex128 spectrum."""
        return self.apply_batch([(sources, positions, looks, out_scale, window)],
                                zero_frequency=zero_frequency, stream=stream)[0]

    def apply_batch(self, items, *, zero_frequency=False, stream=None, mode="fp32"):
        """Several problems (``(sources, positions, looks, out_scale, window)`` each)
        on this table in one set of launches: a list of device (OM, frequency)
        complex128 spectra, each equal to the problem applied alone.

        ``mode``: ``"fp32"`` (CUDA cores), ``"split-bf16"`` or ``"bf16"`` (tensor
        cores, full spectra on a table whose shape fits that path; zero-frequency
        applies and other shapes run on the CUDA cores)."""
        import torch
        lib = _lib.load()
        dev = self.device
        if not items:
            return []
        prepared = [self._prepare(*it, zero_frequency) for it in items]
        host = np.concatenate([np.concatenate([q[k].ravel() for k in ("pts", "rec", "lk", "scale")])
                               for q in prepared])
        d_geom = _lib.upload(host, torch.float64, dev)
        sizes = [q["n_om"] * q["W"] for q in prepared]
        result = torch.empty(max(sum(sizes), 1), dtype=torch.complex128, device=dev)
        probs = (_lib.Ge2Problem * len(prepared))()
        at, r_at = d_geom.data_ptr(), 0
        for i, q in enumerate(prepared):
            probs[i], at = self._problem(q, at, result.data_ptr() + 16 * r_at)
            r_at += sizes[i]
        n = len(prepared)
        if mode not in _lib.MODES:
            raise ValueError(f"unknown contraction mode {mode!r}")
        packed = (self.tc_packed() if mode != "fp32" and not zero_frequency
                  and all(q["W"] == len(self.omega) for q in prepared) else None)
        slots = C.create_string_buffer(int(lib.lh_ge2_batch_slot_bytes(n)))  # pageable staging
        s = _lib.stream_ptr(stream or torch.cuda.current_stream(dev))
        if packed is not None:
            need = int(lib.lh_ge2_tc_workspace_bytes(self.struct, probs, n))
        else:
            need = int(lib.lh_ge2_batch_workspace_bytes(self.struct, probs, n))
        if need == 0:
            raise ValueError("order >=2 problem rejected by the device library")
        if self._workspace is None or self._workspace.numel() < need:
            self._workspace = torch.empty(need, dtype=torch.uint8, device=dev)
        status = None
        if packed is not None:
            status = torch.zeros(1, dtype=torch.int32, device=dev)
            _lib.check(lib.lh_ge2_apply_batch_tc(self.struct, probs, n, _lib.MODES[mode],
                                                 packed.data_ptr(), self._workspace.data_ptr(),
                                                 self._workspace.numel(), slots,
                                                 status.data_ptr(), s), "lh_ge2_apply_batch_tc")
        else:
            _lib.check(lib.lh_ge2_apply_batch(self.struct, probs, n, self._workspace.data_ptr(),
                                              self._workspace.numel(), slots, s),
                       "lh_ge2_apply_batch")
        self.status = status  # LH_STATUS_TIMEOUT when a tensor-core wait gave up
        self._keep = (d_geom, [q["ch"] for q in prepared])  # alive until the stream runs
        out, r_at = [], 0
        for q, size in zip(prepared, sizes):
            out.append(result[r_at:r_at + size].view(q["n_om"], q["W"]))
            r_at += size
        return out


def apply_folded(table: Ge2Table, sources: AxialSources, positions, looks, area, window, *,
                 zero_frequency=False):
    """``shower/ge2.py:99-119``: folded >=2 spectrum (frequency, OM) of node-band sources."""
    if not len(np.atleast_2d(positions)):
        return np.zeros((1 if zero_frequency else len(table.omega), 0), complex)
    return table.apply(sources, positions, looks, np.asarray(area, float), window,
                       zero_frequency=zero_frequency)
