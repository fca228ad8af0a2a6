"""Readout operator: relative spectrum -> time bins as one real matrix.

Reference: ``readout.py:9-72``. ``readout_bins`` refines a spectrum from the
RTE grid (65 nodes) to the readout grid (321) by a not-a-knot cubic spline of
its real and imaginary parts, then ``inverse_bins`` integrates each bin
exactly:

    bins[b] = Re sum_w' K[b, w'] S(w'),
    K[b, w'] = width_b sinc(width_b w' / 2 pi) exp(-i c_b w') weight_w' / pi.

Both steps are linear in the spectrum, so ``W = K @ S_spline`` (bins x 65,
complex) is formed once in float64 on the host, and the device evaluates
``bins = A @ B.T`` with ``A = [Re rel, Im rel]`` and ``B = [Re W, -Im W]``.
"""
from __future__ import annotations

import warnings

import numpy as np

from . import _lib
from .spline import resample_matrix

__all__ = ["readout_matrix", "DeviceReadout"]


def _ceil(a, b):
    return int(-(-int(a) // int(b)))


def _frequency_weights(omega):
    """Trapezoid weights of a half-axis grid (``readout.py:9-15``)."""
    omega = np.asarray(omega, float)
    if (omega.ndim != 1 or len(omega) < 2 or not np.isfinite(omega).all()
            or omega[0] != 0 or np.any(np.diff(omega) <= 0)):
        raise ValueError("Time inversion requires at least two increasing frequencies starting at zero")
    step = np.diff(omega)
    return np.r_[step[0] / 2, (step[:-1] + step[1:]) / 2, step[-1] / 2]


def readout_matrix(omega, edges_ns, readout_omega=None):
    """Complex (bins, len(omega)) operator of ``readout_bins`` (float64)."""
    omega = np.asarray(omega, float)
    edges = np.asarray(edges_ns, float)
    if edges.ndim != 1 or len(edges) < 2 or not np.isfinite(edges).all() or np.any(np.diff(edges) <= 0):
        raise ValueError("Time edges must be finite and strictly increasing")
    grid, spline = omega, np.eye(len(omega))
    if readout_omega is not None and len(omega) > 1:
        readout = np.asarray(readout_omega, float)
        same = len(readout) == len(omega) and np.allclose(readout, omega)
        if not same and np.isclose(readout[-1], omega[-1], rtol=0, atol=1e-12):
            spline = resample_matrix(omega, readout)
            grid = readout
    period = 2 * np.pi / float(np.max(np.diff(grid))) if len(grid) > 1 else np.inf
    if edges[-1] - edges[0] > period * (1 + 1e-9):
        warnings.warn(f"time window of {edges[-1] - edges[0]:g} ns is longer than the "
                      f"{period:g} ns period of the frequency grid; the bins hold repeated "
                      "copies of the waveform (set KernelConfig.readout_omega_per_ns)",
                      RuntimeWarning, stacklevel=2)
    w = _frequency_weights(grid)
    width = np.diff(edges)
    center = (edges[:-1] + edges[1:]) / 2
    kernel = (width[:, None] * np.sinc(width[:, None] * grid / (2 * np.pi))
              * np.exp(-1j * center[:, None] * grid) * (w / np.pi))
    return kernel @ spline


class DeviceReadout:
    """The readout operator resident on the device in every precision layout."""

    def __init__(self, omega, edges_ns, readout_omega=None, *, device="cuda",
                 interleaved_tc=False):
        """``interleaved_tc``: the BF16 operands (``b_hi``, ``b_lo``) take their K
        columns as (Re, Im) per frequency, the layout the fused flash kernel's
        A tile uses; ``b_fp32`` keeps (Re..., Im...)."""
        import torch
        W = readout_matrix(omega, edges_ns, readout_omega)
        n_bins, n_omega = W.shape
        self.n_bins, self.n_omega = int(n_bins), int(n_omega)
        self.k_pad = _ceil(2 * n_omega, 16) * 16
        tiles = _ceil(n_bins, 256)
        self.n_tile = _ceil(_ceil(n_bins, tiles), 16) * 16
        self.n_tiles = _ceil(n_bins, self.n_tile)
        B = np.zeros((n_bins, self.k_pad))
        B[:, :n_omega] = W.real
        B[:, n_omega:2 * n_omega] = -W.imag
        self.matrix = W
        self.b_fp32 = torch.tensor(B, dtype=torch.float32, device=device)
        padded = torch.zeros((self.n_tiles * self.n_tile, self.k_pad), dtype=torch.float32,
                             device=device)
        if interleaved_tc:
            Bi = np.zeros((n_bins, self.k_pad))
            Bi[:, 0:2 * n_omega:2] = W.real
            Bi[:, 1:2 * n_omega:2] = -W.imag
            padded[:n_bins] = torch.tensor(Bi, dtype=torch.float32, device=device)
        else:
            padded[:n_bins] = self.b_fp32
        hi = padded.to(torch.bfloat16)
        lo = (padded - hi.float()).to(torch.bfloat16)

        def tiled(x):  # [tiles][k/8][n_tile][8]
            x = x.reshape(self.n_tiles, self.n_tile, self.k_pad // 8, 8)
            return x.permute(0, 2, 1, 3).contiguous()

        self.b_hi = tiled(hi)
        self.b_lo = tiled(lo)
        self.struct = _lib.ReadoutOperator(
            self.n_bins, self.k_pad, self.n_tile, self.n_tiles, self.b_fp32.data_ptr(),
            self.b_hi.data_ptr(), self.b_lo.data_ptr())

    def packed_bytes(self, mode, rows):
        lib = _lib.load()
        return int(lib.lh_readout_packed_bytes(self.struct, mode, rows))

    def bins(self, relative, *, mode="split-bf16", stream=None):
        """Readout of device spectra ``relative`` (rows, n_omega) complex64 -> (rows, bins)."""
        import torch
        lib = _lib.load()
        m = _lib.MODES[mode]
        rel = torch.view_as_real(relative.to(torch.complex64).contiguous()).contiguous()
        rows = rel.shape[0]
        packed = torch.empty(self.packed_bytes(m, rows), dtype=torch.uint8, device=rel.device)
        out = torch.empty((rows, self.n_bins), dtype=torch.float32, device=rel.device)
        status = torch.zeros(4, dtype=torch.int32, device=rel.device)
        s = _lib.stream_ptr(stream or torch.cuda.current_stream(rel.device))
        _lib.check(lib.lh_readout_pack(self.struct, m, _lib.ptr(rel), self.n_omega, rows,
                                       _lib.ptr(packed), s), "lh_readout_pack")
        _lib.check(lib.lh_readout_rows(self.struct, m, _lib.ptr(packed), rows, _lib.ptr(out),
                                       self.n_bins, _lib.ptr(status), s), "lh_readout_rows")
        return out, status
