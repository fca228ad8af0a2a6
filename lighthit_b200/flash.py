"""Isotropic calibration flashes on the B200: the ``TransportKernel.transport`` path.

Reference: ``TransportKernel._transport_isotropic`` (``transport.py:1061-1164``)
for the centre-ray receiver (``KernelConfig.scattered_receiver == 'centre'``),
with ``ResponseCache.moments_at`` / ``acceptance_spectrum``
(``cache.py:294-436``) and ``readout_bins`` (``readout.py:43-72``).

The multipole table is built once by the reference (``TransportKernel.build``)
and uploaded read-only: the host detrends it exactly as ``moments_at`` does
(attenuation ``exp(-mu_a r)/(4 pi r^2)`` and, for ``radial_phase='flight'``,
the flight phase), forms the not-a-knot cubic coefficients in log r in
float64 and stores them as complex64 in the layout
``[interval][omega][degree][order][power]``. Everything per flash runs in
``liblh_b200.so``; there is no host fallback.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from .model import C_VACUUM_M_PER_NS, Medium, TransportResponse, acceptance_coefficients
from .readout import DeviceReadout
from .spline import spline_coefficients

__all__ = ["FlashTable", "FlashTransport", "BroadbandFlashTransport", "flash_node_photons"]


@dataclass
class FlashTable:
    """Multipole moments of one wavelength (``ResponseCache``): (omega, r, degree, order)."""
    omega_per_ns: np.ndarray
    radii_m: np.ndarray
    moments: np.ndarray
    medium: Medium
    radial_phase: str
    degree: int

    @classmethod
    def load(cls, path):
        """Table exported from the reference (``tests/golden/make_flash_golden.py``)."""
        z = np.load(path)
        medium = Medium(float(z["absorption_per_m"]), float(z["scattering_per_m"]),
                        float(z["g"]), float(z["group_index"]), float(z["wavelength_nm"]))
        return cls(np.asarray(z["omega_per_ns"], float), np.asarray(z["radii_m"], float),
                   np.asarray(z["moments"]), medium, str(z["radial_phase"]), int(z["degree"]))

    @classmethod
    def from_cache_file(cls, path):
        """From the reference's ``transport-<key>.npz`` (``ResponseCache.save``,
        ``cache.py:485-507``), read without the reference."""
        from .formats import load_response_cache
        return load_response_cache(path)

    @classmethod
    def from_cache(cls, cache):
        """From a reference ``ResponseCache`` object (attributes read by name)."""
        m = cache.medium
        return cls(np.asarray(cache.grid.omega_per_ns, float), np.asarray(cache.grid.radii_m, float),
                   np.asarray(cache.moments), Medium(m.absorption_per_m, m.scattering_per_m, m.g,
                                                     m.group_index, m.wavelength_nm),
                   str(cache.radial_phase), int(cache.degree))

    def spline_table(self, top):
        """Complex (interval, omega, degree, order, power) cubic coefficients in log r."""
        r = self.radii_m
        omega = self.omega_per_ns
        scale = np.exp(-self.medium.absorption_per_m * r) / (4 * np.pi * r ** 2)
        if np.any(scale == 0):
            raise FloatingPointError("Reference amplitude underflow: reduce radius range")
        detrended = self.moments[:, :, :top + 1] / scale[None, :, None, None]
        if self.radial_phase == "flight":
            detrended = detrended * np.exp(
                -1j * omega[:, None] * r[None, :] / self.medium.speed_m_per_ns)[:, :, None, None]
        coef = spline_coefficients(np.log(r), detrended, axis=1)  # (w, j, 4, l, o)
        return np.ascontiguousarray(coef.transpose(1, 0, 3, 4, 2))  # (j, w, l, o, p)


class FlashTransport:
    """Batched device transport of monochromatic isotropic flashes.

    ``detector`` and ``config`` follow the reference's ``DetectorArray`` and
    ``KernelConfig``; ``table`` is a :class:`FlashTable` for the flash
    wavelength. ``mode`` selects the readout precision: ``'split-bf16'``
    (tensor cores, hi+lo BF16, fp32 accumulate), ``'bf16'`` or ``'fp32'``
    (the plain CUDA-core path).
    """

    def __init__(self, detector, config, table, *, device="cuda", mode="split-bf16"):
        import torch
        if getattr(config, "scattered_receiver", "centre") != "centre":
            raise NotImplementedError("only the centre-ray receiver is on the device path")
        self.detector, self.config, self.table = detector, config, table
        self.device = torch.device(device)
        self.mode = mode
        dev = self.device
        alpha = acceptance_coefficients(detector.angular_acceptance, table.degree)
        peak = np.max(np.abs(alpha))
        significant = np.flatnonzero(np.abs(alpha) > 1e-12 * peak) if peak > 0 else []
        top = int(significant[-1]) if len(significant) else 0
        if top > 8:
            raise NotImplementedError("acceptance degree above 8 is not on the device path")
        probe = np.asarray(detector.angular_acceptance(np.linspace(-1.0, 1.0, 65)), float)
        if np.allclose(probe, probe[0], rtol=1e-11, atol=1e-14):
            # transport.py:1084-1089: a constant acceptance switches order 1 to
            # the exact full-HG physical-time integral, not implemented here.
            raise NotImplementedError("constant acceptance (exact order 1) is not on the device path")
        self.alpha, self.top = alpha, top
        self.wavelength_nm = float(table.medium.wavelength_nm)
        self.efficiency = float(detector.spectral_weight(self.wavelength_nm))
        n = len(detector.positions_m)
        area = np.broadcast_to(np.asarray(detector.effective_area_m2, float), (n,))
        omega = np.asarray(config.omega_per_ns, float)
        if (len(omega) != len(table.omega_per_ns)
                or not np.allclose(omega, table.omega_per_ns, rtol=0, atol=1e-12)):
            raise ValueError("table and kernel frequency grids differ")
        low, high = map(float, config.radial_range_m)
        if low < table.radii_m[0] - 1e-9 or high > table.radii_m[-1] + 1e-9:
            raise ValueError("radial_range_m lies outside the table's radii")

        def f64(x):
            return torch.tensor(np.ascontiguousarray(x, float), dtype=torch.float64, device=dev)

        self._om_pos = f64(detector.positions_m)
        self._om_look = f64(detector.orientations)
        self._om_area = f64(area)
        self._alpha = f64(alpha[:top + 1])
        self._omega = f64(omega)
        self._log_r = f64(np.log(table.radii_m))
        # device layout (interval, degree, order, power, omega): omega fastest, so
        # a warp's lanes (consecutive frequencies) read each coefficient coalesced
        coef = np.ascontiguousarray(
            table.spline_table(top).astype(np.complex64).transpose(0, 2, 3, 4, 1))
        self._coef = torch.view_as_real(torch.from_numpy(coef)).contiguous().to(dev)
        self._edges = f64(config.relative_time_edges_ns)
        self.readout = DeviceReadout(omega, config.relative_time_edges_ns,
                                     config.readout_omega_per_ns, device=dev,
                                     interleaved_tc=True)
        medium = table.medium
        self.problem = _lib.FlashProblem(
            n, self._om_pos.data_ptr(), self._om_look.data_ptr(), self._om_area.data_ptr(), top,
            self._alpha.data_ptr(), self.efficiency, len(omega), self._omega.data_ptr(),
            len(table.radii_m), self._log_r.data_ptr(), self._coef.data_ptr(),
            medium.absorption_per_m, medium.extinction_per_m, medium.speed_m_per_ns,
            C_VACUUM_M_PER_NS / medium.group_index, low, high, float(config.threshold_pe),
            len(config.relative_time_edges_ns), self._edges.data_ptr())
        self.n_om, self.n_omega = n, len(omega)
        self.n_bins = len(config.relative_time_edges_ns) - 1
        self._workspace = None

    # ------------------------------------------------------------------ batch API
    def allocate(self, n_flash):
        """Device output buffers for ``n_flash`` flashes (reusable across calls)."""
        import torch
        dev, F, D = self.device, int(n_flash), self.n_om
        return dict(
            spectrum=torch.empty((F, D, self.n_omega, 3), dtype=torch.complex64, device=dev),
            components=torch.empty((F, D, 3, self.n_bins), dtype=torch.float32, device=dev),
            charge=torch.empty((F, D, 3), dtype=torch.float64, device=dev),
            origin=torch.empty((F, D), dtype=torch.float64, device=dev),
            active=torch.empty((F, D), dtype=torch.uint8, device=dev),
            status=torch.zeros(4, dtype=torch.int32, device=dev))

    def workspace_bytes(self, n_flash, mode=None):
        lib = _lib.load()
        m = _lib.MODES[mode or self.mode]
        return int(lib.lh_flash_workspace_bytes(self.problem, self.readout.struct, m, int(n_flash)))

    def launch(self, pos, photons, time_ns, out, *, mode=None, stream=None, workspace=None,
               n_device=None, block_threads=0):
        """Enqueue one batch. ``pos`` (F,3), ``photons`` (F,), ``time_ns`` (F,) are
        float64 device tensors; ``out`` comes from :meth:`allocate`. ``n_device``
        (int32 device scalar) makes the kernel read the flash count on the device,
        as a captured graph replayed for varying batch sizes needs. Nothing syncs."""
        import torch
        lib = _lib.load()
        m = _lib.MODES[mode or self.mode]
        F = int(pos.shape[0])
        need = self.workspace_bytes(F, mode)
        if workspace is None and need:
            if self._workspace is None or self._workspace.numel() < need:
                self._workspace = torch.empty(need, dtype=torch.uint8, device=self.device)
            workspace = self._workspace
        batch = _lib.FlashBatch(
            F, pos.data_ptr(), photons.data_ptr(), time_ns.data_ptr(),
            out["spectrum"].data_ptr(), out["components"].data_ptr(), out["charge"].data_ptr(),
            out["origin"].data_ptr(), out["active"].data_ptr(), out["status"].data_ptr(),
            n_device.data_ptr() if n_device is not None else None, int(block_threads))
        s = _lib.stream_ptr(stream or torch.cuda.current_stream(self.device))
        ws_ptr = workspace.data_ptr() if workspace is not None else None
        ws_bytes = workspace.numel() if workspace is not None else 0
        _lib.check(lib.lh_flash_transport(self.problem, self.readout.struct, m, batch, ws_ptr,
                                          ws_bytes, s), "lh_flash_transport")
        return out

    def run(self, positions, photons, time_ns=None, *, mode=None, stream=None):
        """Synchronous batch from host arrays; returns device outputs and checks errors."""
        import torch
        F = len(positions)
        pos = torch.tensor(np.asarray(positions, float).reshape(F, 3), dtype=torch.float64,
                           device=self.device)
        ph = torch.tensor(np.broadcast_to(np.asarray(photons, float), (F,)).copy(),
                          dtype=torch.float64, device=self.device)
        t = torch.tensor(np.zeros(F) if time_ns is None else
                         np.broadcast_to(np.asarray(time_ns, float), (F,)).copy(),
                         dtype=torch.float64, device=self.device)
        out = self.allocate(F)
        self.launch(pos, ph, t, out, mode=mode, stream=stream)
        torch.cuda.synchronize(self.device)
        self.raise_for_status(out)
        return out

    def raise_for_status(self, out, flash=None):
        """Raise the reference's ``ValueError`` for the device status of a batch."""
        status = out["status"].cpu().numpy()
        flags = int(status[0])
        if flags & _lib.LH_STATUS_TIMEOUT:
            raise RuntimeError("a tensor-core pipeline wait timed out on the device")
        if flags & _lib.LH_STATUS_COINCIDENT:
            raise ValueError("isotropic point source cannot coincide with an OM centre")
        if flags & _lib.LH_STATUS_UNSAFE:
            radius = float(status[2:4].view(np.float64)[0])
            raise ValueError(
                f"{int(status[1])} OMs outside radial_range_m have an absorption-only "
                "estimate above threshold; prepare a cache covering the source-to-OM "
                f"distances (up to {radius:g} m). "
                "point_source_radial_range(detector, source.position_m) gives "
                "the geometric range; validate its numerical resolution separately")

    # ------------------------------------------------------------------ drop-in
    def transport(self, source, *, method="isotropic"):
        """``TransportKernel.transport(IsotropicFlash)``: one flash -> ``TransportResponse``."""
        if getattr(source, "wavelength_nm", None) is None:
            raise ValueError("a broadband flash needs one table per wavelength node: "
                             "BroadbandFlashTransport")
        if not np.isclose(float(source.wavelength_nm), self.wavelength_nm, rtol=0, atol=1e-9):
            raise ValueError("flash wavelength differs from the table's wavelength")
        out = self.run(np.asarray(source.position_m, float)[None, :], [float(source.photons)],
                       [float(source.time_ns)])
        return self.response(out, 0, method=method)

    def response(self, out, index, *, method="isotropic"):
        """Host ``TransportResponse`` of flash ``index`` of a finished batch."""
        spectrum = out["spectrum"][index].cpu().numpy().astype(np.complex128)  # (D, w, 3)
        components = out["components"][index].cpu().numpy().astype(np.float64)  # (D, 3, b)
        active = out["active"][index].cpu().numpy()
        return TransportResponse(
            self.detector, np.asarray(self.config.omega_per_ns, float).copy(),
            np.asarray(self.config.relative_time_edges_ns, float).copy(),
            spectrum.transpose(1, 0, 2), components.transpose(0, 2, 1),
            out["charge"][index].cpu().numpy(), out["origin"][index].cpu().numpy(),
            (active & 1).astype(bool), method,
            {"wavelength_nm": [self.wavelength_nm], "detector_angular_model":
             "exact multipole contraction", "first_order":
             "finite-L directional-acceptance spectrum and Fourier bins",
             "fourier_inverted_orders": [1, 2],
             "radial_range_m": list(map(float, self.config.radial_range_m)),
             "readout_precision": self.mode, "route": "lighthit_b200.flash"})


def flash_node_photons(nodes_nm, weights_nm, photons, spectral_shape):
    """``_flash_nodes`` (``transport.py:1049-1059``): photons of each flash at each
    wavelength node, ``photons * weight * shape / (weight . shape)`` ((node, flash))."""
    nodes = np.asarray(nodes_nm, float)
    weights = np.asarray(weights_nm, float)
    shape = np.asarray(spectral_shape(nodes), float)
    if shape.shape != nodes.shape or not np.isfinite(shape).all() or np.any(shape < 0):
        raise ValueError("flash spectral_shape must return finite nonnegative values")
    norm = float(weights @ shape)
    if norm <= 0:
        raise ValueError("flash spectral_shape has zero integral")
    return np.outer(weights * shape / norm, np.atleast_1d(np.asarray(photons, float)))


class BroadbandFlashTransport:
    """Isotropic flashes with a spectral shape (``IsotropicFlash.broadband``).

    The reference transports them at the kernel's wavelength nodes
    (``transport.py:1049-1164``): node photons ``photons * weight * shape /
    (weight . shape)`` (``_flash_nodes``), every node with its own multipole
    table, attenuation, flight time and order-0 arrival, one OM clock for the
    fastest node, the mask and range check on the sum. Here each node is one
    fused device launch (:class:`FlashTransport` on that node's table, with the
    common clock and no mask of its own) and ``lh_flash_combine`` sums the node
    outputs and sets the mask and range check. ``tables``: one
    :class:`FlashTable` per node, in the order of ``node_wavelengths_nm``.
    """

    def __init__(self, detector, config, tables, node_wavelengths_nm, node_weights_nm, *,
                 device="cuda", mode="split-bf16"):
        import torch
        nodes = np.asarray(node_wavelengths_nm, float)
        if len(tables) != len(nodes) or not 1 <= len(nodes) <= 8:
            raise ValueError("one flash table per wavelength node (at most 8)")
        for t, w in zip(tables, nodes):
            if not np.isclose(float(t.medium.wavelength_nm), w, rtol=0, atol=1e-6):
                raise ValueError("flash tables must follow the node wavelengths")
        self.detector, self.config, self.mode = detector, config, mode
        self.device = torch.device(device)
        self.nodes, self.weights = nodes, np.asarray(node_weights_nm, float)
        self.threshold = float(config.threshold_pe)
        fastest = min(float(t.medium.group_index) for t in tables)
        self.node = []
        for t in tables:
            ft = FlashTransport(detector, config, t, device=device, mode=mode)
            ft.problem.origin_speed = C_VACUUM_M_PER_NS / fastest  # transport.py:1124-1125
            ft.problem.threshold = float("inf")                     # the mask is the sum's
            self.node.append(ft)
        self.problem = _lib.FlashProblem.from_buffer_copy(self.node[0].problem)
        self.problem.threshold = self.threshold
        self.n_om, self.n_omega, self.n_bins = (self.node[0].n_om, self.node[0].n_omega,
                                                self.node[0].n_bins)

    def node_photons(self, photons, spectral_shape):
        """``_flash_nodes`` (``transport.py:1049-1059``): (node, flash) photons."""
        return flash_node_photons(self.nodes, self.weights, photons, spectral_shape)

    def run(self, positions, photons, time_ns, spectral_shape, *, stream=None):
        """A batch of flashes sharing one spectral shape: device outputs (checked)."""
        import torch
        F = len(positions)
        dev = self.device
        pos = torch.tensor(np.asarray(positions, float).reshape(F, 3), dtype=torch.float64,
                           device=dev)
        t = torch.tensor(np.broadcast_to(np.asarray(time_ns, float), (F,)).copy(),
                         dtype=torch.float64, device=dev)
        per_node = self.node_photons(np.broadcast_to(np.asarray(photons, float), (F,)),
                                     spectral_shape)
        ph = [torch.tensor(per_node[n], dtype=torch.float64, device=dev)
              for n in range(len(self.node))]
        outs = [ft.launch(pos, ph[n], t, ft.allocate(F), stream=stream)
                for n, ft in enumerate(self.node)]
        out = self.node[0].allocate(F)
        out["origin"] = outs[0]["origin"]  # every node run wrote the common clock
        nd = _lib.FlashNodes()
        nd.n_nodes = len(self.node)
        for n, (ft, o) in enumerate(zip(self.node, outs)):
            nd.spectrum[n] = o["spectrum"].data_ptr()
            nd.components[n] = o["components"].data_ptr()
            nd.charge[n] = o["charge"].data_ptr()
            nd.photons[n] = ph[n].data_ptr()
            nd.efficiency[n] = ft.efficiency
            nd.absorption[n] = float(ft.table.medium.absorption_per_m)
        batch = _lib.FlashBatch(
            F, pos.data_ptr(), 0, t.data_ptr(), out["spectrum"].data_ptr(),
            out["components"].data_ptr(), out["charge"].data_ptr(), out["origin"].data_ptr(),
            out["active"].data_ptr(), out["status"].data_ptr(), None, 0)
        s = _lib.stream_ptr(stream or torch.cuda.current_stream(dev))
        _lib.check(_lib.load().lh_flash_combine(self.problem, nd, batch, s), "lh_flash_combine")
        torch.cuda.synchronize(dev)
        for o in outs:  # coincident sources and wait timeouts of the node runs
            self.node[0].raise_for_status(o)
        self.node[0].raise_for_status(out)
        return out

    def transport(self, source, *, method="isotropic"):
        """``TransportKernel.transport(IsotropicFlash)`` for a broadband flash."""
        if getattr(source, "spectral_shape", None) is None:
            raise ValueError("BroadbandFlashTransport takes flashes with a spectral_shape")
        out = self.run(np.asarray(source.position_m, float)[None, :], [float(source.photons)],
                       [float(source.time_ns)], source.spectral_shape)
        r = self.node[0].response(out, 0, method=method)
        r.metadata["wavelength_nm"] = self.nodes.tolist()
        return r


def _main(argv=None):
    """``python -m lighthit_b200.flash --flashes N --repeat K``: run the fused
    flash launch on the seed-11 calibration workload (48-OM synthetic array,
    450 nm table, 2-250 m) K times and print the mean CUDA-event time. Used to
    profile one kernel on a chosen batch size."""
    import argparse
    from pathlib import Path

    import torch

    from .model import KernelConfig, synthetic_detector
    from .workloads import flash_positions
    ap = argparse.ArgumentParser()
    ap.add_argument("--flashes", type=int, default=4096)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--mode", default="split-bf16", choices=sorted(_lib.MODES))
    ap.add_argument("--block-threads", type=int, default=0)
    args = ap.parse_args(argv)
    det = synthetic_detector()
    cfg = KernelConfig(omega_per_ns=np.linspace(0, 1.2, 65),
                       readout_omega_per_ns=np.linspace(0, 1.2, 321),
                       relative_time_edges_ns=np.arange(-60.0, 745.0, 5.0),
                       radial_range_m=(2.0, 250.0), threshold_pe=0.01)
    table = FlashTable.load(Path(__file__).resolve().parent / "tables" / "flash_450nm_2-250m.npz")
    ft = FlashTransport(det, cfg, table, device="cuda", mode=args.mode)
    F = args.flashes
    pos = torch.tensor(flash_positions(F, det.positions_m.mean(axis=0), seed=11,
                                       om_positions=det.positions_m), device=ft.device)
    ph = torch.full((F,), 1e10, dtype=torch.float64, device=ft.device)
    tt = torch.zeros(F, dtype=torch.float64, device=ft.device)
    out = ft.allocate(F)
    ft.launch(pos, ph, tt, out, block_threads=args.block_threads)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.repeat):
        ft.launch(pos, ph, tt, out, block_threads=args.block_threads)
    e1.record()
    torch.cuda.synchronize()
    ft.raise_for_status(out)
    ms = e0.elapsed_time(e1) / max(args.repeat, 1)
    print(f"flashes {F} mode {args.mode}: {ms:.4f} ms per launch, "
          f"{F * ft.n_om * (ft.n_omega * 24 + 3 * ft.n_bins * 4 + 33) / ms / 1e6:.1f} GB/s of outputs")


if __name__ == "__main__":
    _main()
