"""Order 0 on the B200: continuous-spectrum direct light to the first glass entry.

Reference: ``PreparedBallistic`` (``_surface_ballistic.py:20-118``) as
``transport_prompt`` uses it for ``ballistic_method="first-entry"``
(``prompt.py:640-660`` charge of every OM within reach, ``prompt.py:896-903``
charge and bins of the active OMs). The device evaluates the reference's
direct ray form (``_surface_ballistic_rays.evaluate``) over the candidate
pairs of ``interval_candidates`` at a fixed Gauss order (8 by default; the
reference's own adaptive rule reaches ``1e-10 + 2e-6 |q|`` and order 8 agrees
with it to ~1e-7 in charge).

The optical panels are ``prepare_optics(kernel, config, exact_response=True)``
(``ballistic_interval.py:64-161``): built once on the host by the reference
and uploaded read-only with the detector arrays (``Order0Optics``).
"""
from __future__ import annotations

import numpy as np

from . import _lib

__all__ = ["Order0Optics", "DirectLight", "ElementBatch", "ResidentElements", "order0",
           "ELEMENT_FIELDS",
           "OPTICS_FIELDS"]

ELEMENT_FIELDS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
                  "start_ns", "end_ns")
OPTICS_FIELDS = ("panel_edges", "phase_nodes", "group_nodes", "extinction_nodes",
                 "efficiency_coefficients")
CHARGE_ONLY_EDGES = np.array([-1e100, 1e100])

_ERRORS = [(_lib.LH_STATUS_INSIDE_GLASS, "emitting segment intersects the glass boundary"),
           (_lib.LH_STATUS_ON_TRACK, "point receiver lies on emitting track: singular "
                                     "ballistic fluence"),
           (_lib.LH_STATUS_NEGATIVE_ACCEPTANCE, "negative ballistic angular response"),
           (_lib.LH_STATUS_OVERFLOW, "ballistic bin cuts exceed the kernel's per-range "
                                     "capacity; use coarser bins")]


def _field(source, name):
    return source[name] if isinstance(source, dict) else getattr(source, name)


class Order0Optics:
    """Optical panels, acceptance and OM spheres resident on the device."""

    def __init__(self, optics, positions_m, looks, areas_m2, radii_m, alpha, *, order=8,
                 check_order=0, device="cuda"):
        """``check_order``: a lower Gauss order evaluated beside ``order`` when a
        call asks for an error estimate (0: none)."""
        import torch
        self.device = torch.device(device)
        positions = np.ascontiguousarray(np.atleast_2d(positions_m), float)
        n = len(positions)
        self.n_om = n
        self.order = int(order)
        self.check_order = int(check_order)
        self._source = (optics, positions, looks, areas_m2, radii_m, alpha)
        radii = np.broadcast_to(np.asarray(radii_m, float), (n,))
        if np.any(radii <= 0):
            raise ValueError("the first-entry order 0 needs OM sphere radii > 0")
        arrays = dict(
            om_pos=positions, om_look=np.ascontiguousarray(np.atleast_2d(looks), float),
            om_area=np.broadcast_to(np.asarray(areas_m2, float), (n,)),
            om_radius=radii, alpha=np.asarray(alpha, float),
            panel_edges=optics["panel_edges"], phase=optics["phase_nodes"],
            group=optics["group_nodes"], extinction=optics["extinction_nodes"],
            efficiency=optics["efficiency_coefficients"])
        gx, gw = np.polynomial.legendre.leggauss(self.order)
        cx, cw = (np.polynomial.legendre.leggauss(self.check_order) if self.check_order
                  else (np.zeros(1), np.zeros(1)))
        arrays.update(gauss_x=gx, gauss_w=gw, check_x=cx, check_w=cw)
        self._t = {k: torch.tensor(np.ascontiguousarray(v, float), dtype=torch.float64,
                                   device=self.device) for k, v in arrays.items()}
        eff = np.asarray(optics["efficiency_coefficients"], float)
        t = self._t
        self.struct = _lib.Order0Optics(
            n, t["om_pos"].data_ptr(), t["om_look"].data_ptr(), t["om_area"].data_ptr(),
            t["om_radius"].data_ptr(), len(arrays["alpha"]), t["alpha"].data_ptr(),
            len(optics["panel_edges"]), t["panel_edges"].data_ptr(), t["phase"].data_ptr(),
            t["group"].data_ptr(), t["extinction"].data_ptr(), eff.shape[1],
            t["efficiency"].data_ptr(), self.order, t["gauss_x"].data_ptr(),
            t["gauss_w"].data_ptr(), self.check_order, t["check_x"].data_ptr(),
            t["check_w"].data_ptr())

    def subset(self, ids, *, order):
        """These optics for the OMs ``ids`` at Gauss ``order`` (no check order)."""
        optics, positions, looks, areas, radii, alpha = self._source
        n = len(positions)
        ids = np.asarray(ids, np.int64)
        return Order0Optics(optics, positions[ids], np.atleast_2d(looks)[ids],
                            np.broadcast_to(np.asarray(areas, float), (n,))[ids],
                            np.broadcast_to(np.asarray(radii, float), (n,))[ids], alpha,
                            order=order, device=self.device)

    def workspace(self, nbytes):
        """Device scratch of at least ``nbytes`` (kept and grown across calls)."""
        import torch
        if getattr(self, "_workspace", None) is None or self._workspace.numel() < nbytes:
            self._workspace = torch.empty(max(int(nbytes), 1), dtype=torch.uint8,
                                          device=self.device)
        return self._workspace

    @classmethod
    def from_arrays(cls, d, **kw):
        """From a dict holding the optics fields and the detector arrays."""
        return cls({k: d[k] for k in OPTICS_FIELDS}, d["positions_m"], d["looks"], d["areas_m2"],
                   d["radii_m"], d["alpha"], **kw)

    @classmethod
    def from_kernel(cls, kernel, **kw):
        """Tables built by the reference for its ``TransportKernel`` (host, once)."""
        from lighthit.ballistic_interval import BallisticIntervalConfig, prepare_optics
        optics = prepare_optics(kernel, BallisticIntervalConfig(), exact_response=True)
        d = kernel.detector
        n = len(d)
        return cls(optics, d.positions_m, -np.asarray(d.orientations, float),
                   np.broadcast_to(np.asarray(d.effective_area_m2, float), (n,)),
                   np.broadcast_to(np.asarray(d.receiver_surface.radii(n), float), (n,)),
                   kernel.acceptance()["alpha"], **kw)


class ResidentElements(dict):
    """One source's element arrays on the host (which the route's host logic
    reads: delay groups, frames, selection) and already in device memory (which
    its kernels read), uploaded once when the source is created."""

    def __init__(self, elements, device):
        import torch
        super().__init__((k, np.ascontiguousarray(_field(elements, k), float))
                         for k in ELEMENT_FIELDS)
        self.device_arrays = {k: torch.tensor(v, dtype=torch.float64, device=device)
                              for k, v in self.items()}


class ElementBatch:
    """Elements of several events, concatenated on the device in one upload.

    ``event(k)`` gives device views of event ``k``'s arrays (no copy), so the
    other stages of a route read the same upload.
    """

    WIDTH = {"start_m": 3, "direction": 3}

    def __init__(self, events, device):
        import torch
        counts = np.array([len(np.atleast_1d(_field(e, "length_m"))) for e in events], np.int64)
        self.n_events = len(events)
        self.counts = counts
        offsets = np.zeros(len(events) + 1, np.int64)
        offsets[1:] = np.cumsum(counts)
        self.offsets = offsets
        self.n_elements = n = int(offsets[-1])
        if events and all(isinstance(e, ResidentElements) for e in events):
            # already on the device: one concatenation there, only the offsets travel
            flat = torch.cat([e.device_arrays[name].reshape(-1) for name in ELEMENT_FIELDS
                              for e in events]
                             + [_lib.upload(offsets.astype(float), torch.float64, device)])
        else:
            parts = [_field(e, name) for name in ELEMENT_FIELDS for e in events]
            flat, _ = _lib.upload_parts(parts + [offsets], torch.float64, device)
        self._t = {}
        pos = 0
        for name in ELEMENT_FIELDS:
            w = self.WIDTH.get(name, 1)
            view = flat[pos:pos + n * w]
            self._t[name] = view.view(n, w) if w > 1 else view
            pos += n * w
        self._t["offsets"] = flat[pos:].to(torch.int64)
        self._flat = flat

    def pointers(self):
        t = self._t
        return [t[k].data_ptr() for k in ELEMENT_FIELDS]

    def event(self, k):
        """Device views of event ``k``'s element arrays (reference field names)."""
        a, b = int(self.offsets[k]), int(self.offsets[k + 1])
        return {name: self._t[name][a:b] for name in ELEMENT_FIELDS}


def order0(optics: Order0Optics, events, origins=None, edges=None, *, stream=None,
           check=True, estimate=False):
    """Order-0 charge (events, OMs) and bins (events, OMs, bins) on the device.

    ``events``: element sets (reference ``SpectralLightElements`` or dicts with
    its field names), already cut at the spectral threshold as the route does
    (``prompt.py:542-562``). ``edges`` None gives the charge only
    (``PreparedBallistic.charge``); otherwise ``origins`` (events, OMs) are the
    per-OM clocks and the bins are ``PreparedBallistic.bins`` for every OM.
    ``estimate``: also the charge at the optics' check order (``charge_check``).
    """
    import torch
    dev = optics.device
    batch = events if isinstance(events, ElementBatch) else ElementBatch(list(events), dev)
    E, n = batch.n_events, optics.n_om
    want_bins = edges is not None
    edges_np = np.asarray(edges if want_bins else CHARGE_ONLY_EDGES, float)
    if edges_np.ndim != 1 or len(edges_np) < 2 or np.any(np.diff(edges_np) <= 0):
        raise ValueError("invalid time origins or edges")
    if origins is None:
        if want_bins:
            raise ValueError("bins need per-OM time origins")
        origins_t = torch.zeros((E, n), dtype=torch.float64, device=dev)
    else:
        origins_t = (origins.to(dev, torch.float64).contiguous()
                     if isinstance(origins, torch.Tensor) else
                     _lib.upload(np.broadcast_to(np.asarray(origins, float), (E, n)),
                                 torch.float64, dev))
    edges_t = _lib.upload(edges_np, torch.float64, dev)
    charge = torch.empty((E, n), dtype=torch.float64, device=dev)
    bins = (torch.empty((E, n, len(edges_np) - 1), dtype=torch.float64, device=dev)
            if want_bins else None)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    charge_check = (torch.empty((E, n), dtype=torch.float64, device=dev)
                    if estimate and optics.check_order > 0 else None)
    t = batch._t
    b = _lib.Order0Batch(E, t["offsets"].data_ptr(), batch.n_elements, *batch.pointers(),
                         origins_t.data_ptr(), len(edges_np), edges_t.data_ptr(),
                         charge.data_ptr(), bins.data_ptr() if bins is not None else None,
                         status.data_ptr(), None, 0,
                         charge_check.data_ptr() if charge_check is not None else None)
    lib = _lib.load()
    need = int(lib.lh_order0_workspace_bytes(optics.struct, b))
    if need == 0:
        raise ValueError("order-0 problem rejected by the device library")
    workspace = optics.workspace(need)
    b.workspace, b.workspace_bytes = workspace.data_ptr(), workspace.numel()
    s = _lib.stream_ptr(stream or torch.cuda.current_stream(dev))
    _lib.check(lib.lh_order0(optics.struct, b, s), "lh_order0")
    result = dict(charge=charge, bins=bins, status=status, charge_check=charge_check,
                  _keep=(batch, origins_t, edges_t, workspace))
    if check:
        raise_status(int(status.item()))
    return result


def raise_status(flags):
    """The reference's ValueError for a device status word."""
    for bit, message in _ERRORS:
        if flags & bit:
            raise ValueError(message)


class DirectLight:
    """``PreparedBallistic`` for one element set (first-entry sphere mode)."""

    def __init__(self, optics: Order0Optics, source):
        beta = np.asarray(_field(source, "beta"), float)
        c0 = np.asarray(_field(source, "coefficient0"), float)
        c2 = np.asarray(_field(source, "coefficient2"), float)
        # _surface_ballistic.py:24-27
        if not np.allclose(c2, -c0 / beta ** 2, rtol=1e-10, atol=1e-20):
            raise ValueError("source must have the physical Cherenkov C0/C2/beta relation")
        self.optics = optics
        self.source = source
        self._batch = ElementBatch([source], optics.device)
        self.cached_charge = None

    def charge(self):
        if self.cached_charge is None:
            self.cached_charge = order0(self.optics, self._batch)["charge"][0].cpu().numpy()
        return self.cached_charge

    def bins(self, ids, origins, edges):
        """Charge and bins of the OMs ``ids`` (``_surface_ballistic.py:106-118``)."""
        ids = np.asarray(ids, dtype=np.int64)
        origins, edges = np.asarray(origins, float), np.asarray(edges, float)
        if (origins.shape != (len(ids),) or not np.isfinite(origins).all()
                or edges.ndim != 1 or len(edges) < 2 or not np.isfinite(edges).all()
                or np.any(np.diff(edges) <= 0)):
            raise ValueError("invalid time origins or edges")
        full = np.zeros(self.optics.n_om)
        full[ids] = origins
        out = order0(self.optics, self._batch, full[None], edges)
        return out["charge"][0, ids].cpu().numpy(), out["bins"][0, ids].cpu().numpy()
