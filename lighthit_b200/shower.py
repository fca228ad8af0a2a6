"""The shower route on the B200: ``ShowerTransport`` with every order on the device.

Reference: ``transport_shower`` (``shower/api.py:321-637``) behind
``ShowerTransport.__call__`` (``shower/api.py:213-318``). The call surface, the
selection algebra and the response fields are the reference's; the numerics
are the device kernels of this package:

* order 0: ``order0`` (first-entry ray quadrature, ``lh_order0``);
* order 1: ``order1`` (pencil compression + grouped pencils, ``lh_order1_*``);
* order >=2: ``source`` (axial-slice node-band sources, ``lh_source_compile``)
  contracted by ``ge2`` (``lh_ge2_apply``) at the zero frequency (predictor,
  exact candidates) and at all frequencies (active OMs);
* readout of the >=2 spectrum to the time bins: ``readout`` (``lh_readout_*``);
* clocks and module selection: ``lh_om_geometry`` (float64, bit-identical);
* element portions closer to an OM than the tables' radial minimum: the
  near-field clamp of ``near`` (``lh_near_field``, ``near_field.py:91-217``).

Tables are built once by the reference and stored under ``tables/``
(``build_tables.py``): the folded >=2 kernels, the first radial interval of the
per-wavelength kernels (near field) and the route's medium and detector
constants. Elements above the Cherenkov threshold in only some bands run as
the reference's per-band order-1 units and per-band source lattices; receiver
subsets (``receivers=``) run on ``ShowerTables.subset``. A table without its
near-field file raises ``NotImplementedError`` when a shower needs the clamp.
Order 1 follows the reference's global screen (``prompt.py:720-812``): a
coarse charge pass for every OM in reach (``compress_screen``/``screen_order1``,
``_prompt_screen.py``: 2 m cells, 24 ring nodes, 8-pixel parent faces refined
to 32-pixel children near each OM, a two-node radial rule, charge batches
without emission time), full resolution where ``q0 + extra + 3 q1_coarse``
reaches threshold, widened when the coarse pass underestimated. Coarse-only
OMs keep the coarse charge, as in the reference.
"""
from __future__ import annotations

import ctypes as C
import functools
from contextlib import contextmanager
from dataclasses import dataclass, field
from pathlib import Path
from time import perf_counter

import numpy as np

from . import _lib
from .ge2 import AxialSources, Ge2Table
from .order0 import (ElementBatch, Order0Optics, ResidentElements, order0,
                     raise_status as raise_order0_status)
from .near import NearTable, add_near_field
from .order1 import (Order1Tables, PromptSettings, acceptance_monomials, element_box, grouped,
                     grouped_widening, pencils)
from .readout import DeviceReadout
from .source import ShowerBasisSettings, SourceCompiler, axis_frame

__all__ = ["ShowerSettings", "ShowerTables", "ShowerTransport", "HybridTransportResponse"]

C_M_PER_NS = 0.299792458
UNFUSED_PIXEL_FACE, UNFUSED_RING_NODES = 32, 96  # PromptConfig defaults (prompt.py:172-173)
TABLES = Path(__file__).resolve().parent / "tables"
ELEMENT_FIELDS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
                  "start_ns", "end_ns")


@dataclass(frozen=True)
class ShowerSettings:
    """``ShowerConfig`` fields the route reads (``shower/api.py:47-90``)."""
    predictor_cell_m: float = 2.0
    predictor_safety: float = 2.0
    prompt_delay_ns: float = 20.0
    delayed_cell_ns: float = 20.0        # ShowerConfig.delayed_cell_ns
    min_distance_m: float = 0.1          # PromptConfig.min_distance_m
    readout_mode: str = "split-bf16"
    # The >=2 contraction of the full spectra: "split-bf16" or "bf16" on the
    # tensor cores (BF16 operands, float32 accumulation), "fp32" on the CUDA cores.
    contraction_mode: str = "split-bf16"
    # Gauss order of the order-0 ray quadrature (wavelength, along-track and
    # azimuth nodes per piece). Against the reference's control-variate order 0
    # on the README shower: order 6 agrees to 6e-8 in charge (order 8: 2.5e-8,
    # order 5: 4.6e-7), inside the reference's own tolerance 1e-10 + 2e-6 |q|
    # (_surface_ballistic.py:149-168), at (6/8)^3 of order 8's work.
    order0_gauss: int = 6
    # Error estimate of order 0: the charge at this lower Gauss order is formed
    # in the same launch. Their difference bounds the lower order's error, and
    # order 6's error is several times smaller still (on the README shower
    # order 5 agrees with the reference's order 0 to 4.6e-7, order 6 to 6e-8), so
    # an OM passes when the difference is within the reference's tolerance
    # 1e-10 + 2e-6 |q| (BallisticIntervalConfig, ballistic_interval.py:31-36).
    # An OM that does not is evaluated again with the order doubled until
    # successive charges agree within a quarter of that tolerance (the
    # reference's adaptive loop, _surface_ballistic.py:179-229), and raises the
    # reference's ValueError at order0_max_order (_surface_ballistic.py:195-196).
    # 0 skips the estimate.
    order0_check: int = 5
    order0_max_order: int = 64
    order0_relative_tolerance: float = 2e-6
    order0_absolute_tolerance_pe: float = 1e-10
    # The device integrand is float32 with hardware sine/exponential (absolute
    # error near 2^-21 per node), so two quadrature orders of one OM can differ
    # by ~1e-6 of its charge however far the order is raised. Differences below
    # this fraction of the charge are taken as that float32 floor rather than
    # as quadrature error (the route's order-0 charge agrees with the
    # reference's float64 to a few 1e-6); 0 tests the reference's tolerance alone.
    order0_float32_floor: float = 1e-5
    screen: bool = True                  # PromptConfig.screen
    screen_margin: float = 3.0           # PromptConfig.screen_margin


@dataclass
class HybridTransportResponse:
    """The reference's ``HybridTransportResponse`` fields (``transport.py:331-383``)."""
    detector: object
    omega_per_ns: np.ndarray
    relative_time_edges_ns: np.ndarray
    spectrum_ge2_pe: np.ndarray
    components_pe: np.ndarray
    charge_components_pe: np.ndarray
    time_origin_ns: np.ndarray
    active: np.ndarray
    method: str
    metadata: dict = field(default_factory=dict)

    @property
    def charge_pe(self):
        return self.charge_components_pe.sum(axis=1)

    @property
    def bins_pe(self):
        return self.components_pe.sum(axis=2)


class ShowerTables:
    """Everything the route reads, resident on the device (built once)."""

    def __init__(self, route, folded, *, near=None, device="cuda", settings=ShowerSettings()):
        import torch
        self.device = torch.device(device)
        r = dict(np.load(route)) if not isinstance(route, dict) else route
        self.positions = np.ascontiguousarray(r["positions_m"], float)
        n = len(self.positions)
        self.looks = np.ascontiguousarray(r["looks"], float)
        self.areas = np.ascontiguousarray(r["areas_m2"], float)
        self.radii = np.ascontiguousarray(r["radii_m"], float)
        self.alpha = np.asarray(r["alpha"], float)
        self.omega = np.asarray(r["omega_per_ns"], float)
        self.readout_omega = np.asarray(r["readout_omega_per_ns"], float)
        self.edges = np.asarray(r["edges_ns"], float)
        self.threshold = float(r["threshold_pe"])
        self.radial = tuple(float(v) for v in r["radial_range_m"])
        self.wavelengths = np.asarray(r["wavelength_nm"], float)
        self.weights = np.asarray(r["weight_nm"], float)
        self.phase = np.asarray(r["phase_index"], float)
        self.group = np.asarray(r["group_index"], float)
        self.absorption = np.asarray(r["absorption_per_m"], float)
        self.efficiency = np.asarray(r["efficiency"], float)
        self.threshold_phase = float(r["threshold_phase"])
        self.peak_acceptance = float(r["peak_acceptance"])
        self.fold_bands = np.asarray(r["fold_bands"], np.int64)
        self.fold_scale = np.asarray(r["fold_scale"], float)
        self.fold_phase = np.asarray(r["fold_phase"], float)
        self.prompt = {k: np.asarray(r[k], float) for k in ("mus", "mut", "speed", "s0w", "s2w")}
        self.g = float(r["g"])
        self.source_degree = int(r["source_degree"])
        self.azimuthal_degree = int(r["azimuthal_degree"])
        self.settings = settings
        self._optics = {k: np.asarray(r[f"optics_{k}"], float) for k in (
            "panel_edges", "phase_nodes", "group_nodes", "extinction_nodes",
            "efficiency_coefficients")}
        self._om_tables()
        bands = self.fold_bands
        self.source = SourceCompiler(self.wavelengths[bands], self.fold_phase[bands],
                                     self.fold_scale[bands], self.source_degree,
                                     self.azimuthal_degree, self.omega,
                                     settings=ShowerBasisSettings(), device=device)
        fold = dict(np.load(folded)) if not isinstance(folded, dict) else folded
        self.ge2 = Ge2Table(fold, self.alpha, source_degree=self.source_degree,
                            azimuthal_degree=self.azimuthal_degree, device=device)
        if not np.allclose(self.ge2.omega, self.omega, rtol=0, atol=1e-12):
            raise ValueError("folded >=2 kernels and route frequencies differ")
        low_c, high_c = self.ge2.radial_limits()
        if self.radial[0] < low_c - 1e-9 or self.radial[1] > high_c + 1e-9:
            raise ValueError("radial window must lie inside the kernel cache")
        self.readout = DeviceReadout(self.omega, self.edges, self.readout_omega, device=device)
        self._shifted_readout = {}
        # near-field clamp (near_field.py:91-171): the first radial interval of
        # every wavelength's order >=2 spline
        self.near = None if near is None else NearTable(
            near, wavelength_nm=self.wavelengths, weight_nm=self.weights,
            efficiency=self.efficiency, phase_index=self.phase, alpha=self.alpha, device=device)
        if self.near is not None and (
                not np.allclose(self.near.omega, self.omega, rtol=0, atol=1e-12)
                or abs(self.near.radial_minimum - self.radial[0]) > 1e-9 * self.radial[0]):
            raise ValueError("near-field table and route frequencies or radial minimum differ")
        # spectral_attenuation (shower_basis.py:388-405) for the far-tail screen
        w = self.weights * self.efficiency / self.wavelengths ** 2
        lowest = float(self.absorption.min())
        radius = np.geomspace(1e-3, 1e5, 1025)
        log_factor = (np.log(np.exp(-np.outer(radius, self.absorption - lowest)) @ w / w.sum())
                      - lowest * radius)
        self._attenuation = (radius, log_factor)
        self._att = (torch.tensor(radius, dtype=torch.float64, device=self.device),
                     torch.tensor(log_factor, dtype=torch.float64, device=self.device))
        self._window_ws = None
        self.n_om = n

    def _om_tables(self):
        """The OM-dependent device tables (orders 0 and 1, OM arrays)."""
        import torch
        dev, settings = self.device, self.settings
        self.order0 = Order0Optics(self._optics, self.positions, self.looks, self.areas,
                                   self.radii, self.alpha, order=settings.order0_gauss,
                                   check_order=settings.order0_check, device=dev)
        self.order1 = Order1Tables(self.prompt, self.g, acceptance_monomials(self.alpha),
                                   self.positions, self.looks, self.areas, self.edges,
                                   settings=PromptSettings(), device=dev)
        self.order1_screen = Order1Tables(self.prompt, self.g, acceptance_monomials(self.alpha),
                                          self.positions, self.looks, self.areas, self.edges,
                                          settings=PromptSettings().coarse(), compute_bins=False,
                                          device=dev)
        self._order1_bands = {}
        self._pos = torch.tensor(self.positions, dtype=torch.float64, device=dev)
        self._looks = torch.tensor(self.looks, dtype=torch.float64, device=dev)
        self._areas = torch.tensor(self.areas, dtype=torch.float64, device=dev)
        self._window_ws = None
        self.n_om = len(self.positions)

    def subset(self, receivers):
        """These tables for the OMs ``receivers`` only, with threshold zero
        (``subset_kernel`` in ``ShowerTransport._event``, ``shower/api.py:205-212``):
        the OM-independent device tables (>=2 kernels, source compiler, readout,
        near field) are shared, the OM tables rebuilt for the subset."""
        import copy
        ids = np.asarray(receivers, np.int64).ravel()
        if not len(ids) or ids.min() < 0 or ids.max() >= self.n_om or len(np.unique(ids)) != len(ids):
            raise ValueError("receivers must be distinct OM indices of the detector")
        view = copy.copy(self)
        view.positions = np.ascontiguousarray(self.positions[ids])
        view.looks = np.ascontiguousarray(self.looks[ids])
        view.areas = np.ascontiguousarray(self.areas[ids])
        view.radii = np.ascontiguousarray(self.radii[ids])
        view.threshold = 0.0
        view.receivers = ids
        view._om_tables()
        return view

    @classmethod
    def from_reference(cls, kernel, data=None, *, config=None, **kw):
        """Tables of a reference ``TransportKernel`` and its prepared shower data
        (``ShowerData``, a manifest path, or None to search next to the kernel's
        cache), read through the reference's own ``ShowerTransport``
        (``shower/api.py:124-174``): the folded order >=2 kernels, the
        near-field interval and the route constants, uploaded once. Needs the
        reference package; the device route reads nothing of it afterwards."""
        from lighthit.shower import ShowerTransport as ReferenceRoute
        from .tables.build_tables import folded_kernels, near_interval, route_constants
        route = ReferenceRoute(kernel, data, config=config)
        tables = route.tables()
        return cls(route_constants(route, tables), folded_kernels(route, tables),
                   near=near_interval(route, tables), **kw)

    @classmethod
    def from_packs(cls, route, folded_pack, kernel_pack=None, **kw):
        """Tables from the reference's own files, without the reference: the
        route constants (``route``: a ``route_<config>.npz`` or its dict), the
        band-folded order >=2 directory ``ShowerData.ge2_band_fold`` points to
        (``folded.npy`` + ``folded.json``), and optionally the per-wavelength
        kernel pack of ``ShowerData.ge2_pack`` (``pack.json`` + ``<n>.npy``),
        whose bundle on the route's frequencies gives the near-field interval
        (``lighthit_b200.formats``)."""
        from .formats import load_folded_pack, load_kernel_pack, near_table
        folded = load_folded_pack(folded_pack)
        near = kw.pop("near", None)
        if kernel_pack is not None:
            omega = np.asarray(folded["omega"], float)
            for bundle in load_kernel_pack(kernel_pack).values():
                if (len(bundle["omega"]) == len(omega)
                        and np.allclose(bundle["omega"], omega, rtol=0, atol=1e-12)):
                    near = near_table(bundle)
                    break
            else:
                raise ValueError("the kernel pack holds no bundle on the folded frequencies")
        return cls(route, folded, near=near, **kw)

    @classmethod
    def synthetic(cls, name="c0", **kw):
        """Synthetic Baikal-like workloads: ``c0`` (48 OMs, 2-150 m), ``c2`` (384 OMs,
        2-450 m), ``c3`` (384 OMs, 1-300 m, 8 wavelength nodes, degree 16, azimuthal
        degree 4, 1025 readout nodes, 1 ns bins to 2000 ns)."""
        folded = {"c0": "ge2_fold_48om_2-150m.npz", "c2": "ge2_fold_384om_2-450m.npz",
                  "c3": "ge2_fold_384om_1-300m.npz"}
        if name not in folded:
            raise ValueError("known synthetic tables: c0, c2, c3")
        near = TABLES / f"near_{name}.npz"
        kw.setdefault("near", near if near.exists() else None)
        return cls(TABLES / f"route_{name}.npz", TABLES / folded[name], **kw)

    def om_geometry_batch(self, prompt_store, store, group_index, *, host=True):
        """Per shower: distances to the prompt elements and earliest arrivals
        (host arrays, or the device tensors with ``host=False``)."""
        import torch
        dev = self.device
        n = self.n_om
        out = []
        for batch, want_distance in ((prompt_store, True), (store, False)):
            t = batch._t
            res = torch.empty((batch.n_events, n), dtype=torch.float64, device=dev)
            g = _lib.OmGeometry(n, self._pos.data_ptr(), batch.n_events, t["offsets"].data_ptr(),
                                t["start_m"].data_ptr(), t["direction"].data_ptr(),
                                t["length_m"].data_ptr(), t["start_ns"].data_ptr(),
                                float(group_index), res.data_ptr() if want_distance else None,
                                None if want_distance else res.data_ptr())
            sp = _lib.stream_ptr(torch.cuda.current_stream(dev))
            _lib.check(_lib.load().lh_om_geometry(C.byref(g), sp), "lh_om_geometry")
            out.append(res)
        return tuple(_lib.fetch(out)) if host else tuple(out)

    def order1_band(self, band, *, coarse=False):
        """Order-1 tables of one wavelength band for the per-band units (elements
        above threshold in only some bands): that band's constants and the
        unfused pencil resolution ``PromptConfig.pixel_face`` / ``ring_nodes``
        (``prompt.py:172-173``), or the coarse screen's (built once)."""
        key = (int(band), bool(coarse))
        if key not in self._order1_bands:
            from dataclasses import replace
            settings = replace(PromptSettings(), pixel_face=UNFUSED_PIXEL_FACE,
                               ring_nodes=UNFUSED_RING_NODES)
            self._order1_bands[key] = Order1Tables(
                {k: v[band:band + 1] for k, v in self.prompt.items()}, self.g,
                acceptance_monomials(self.alpha), self.positions, self.looks, self.areas,
                self.edges, settings=settings.coarse() if coarse else settings,
                compute_bins=not coarse, device=self.device)
        return self._order1_bands[key]

    def readout_shifted(self, shift_ns):
        """The readout operator on the window edges seen from a delay ``shift_ns``
        (``edges - shift``: a delayed group's light read on its own clock)."""
        key = float(shift_ns)
        if key not in self._shifted_readout:
            self._shifted_readout[key] = DeviceReadout(self.omega, self.edges - key,
                                                       self.readout_omega, device=self.device)
        return self._shifted_readout[key]

    def radial_window(self, compiled):
        """Per (event, node band, OM): basis points inside / beyond the radial range
        and the far-tail photon sum, for compiled sources ``(points, channels,
        n_points (host), frame)`` (device points and channels): three host arrays."""
        import torch
        dev = self.device
        n, nb, ne = self.n_om, len(self.fold_bands), len(compiled)
        events = (_lib.WindowEvent * ne)()
        for e, (points, channels, npts, frame) in enumerate(compiled):
            E = events[e]
            for b in range(nb):
                E.n_points[b] = int(npts[b])
            E.capacity = int(points.shape[1])
            E.points, E.channels = points.data_ptr(), channels.data_ptr()
            E.channel_stride = 2 * int(channels.shape[2]) * int(channels.shape[3])
            centre, axis, first, second = frame
            for k in range(3):
                E.centre[k], E.axis[k] = float(centre[k]), float(axis[k])
                E.first[k], E.second[k] = float(first[k]), float(second[k])
        cells = ne * nb * n
        out = torch.empty(16 * cells, dtype=torch.uint8, device=dev)  # n_near, n_far, far_sum
        S = _lib.RadialWindowProblem()
        S.n_om, S.n_bands, S.om_pos = n, nb, self._pos.data_ptr()
        S.radial_low, S.radial_high = self.radial
        S.n_att, S.att_radius, S.att_log = len(self._attenuation[0]), self._att[0].data_ptr(), \
            self._att[1].data_ptr()
        S.photon_scale = float(np.sqrt(4 * np.pi))
        for b, band in enumerate(self.fold_bands):
            S.efficiency[b] = float(self.efficiency[band])
        S.n_near, S.n_far, S.far_sum = (out.data_ptr(), out.data_ptr() + 4 * cells,
                                        out.data_ptr() + 8 * cells)
        lib = _lib.load()
        need = int(lib.lh_window_slot_bytes(ne))
        if self._window_ws is None or self._window_ws.numel() < need:
            self._window_ws = torch.empty(need, dtype=torch.uint8, device=dev)
        sp = _lib.stream_ptr(torch.cuda.current_stream(dev))
        _lib.check(lib.lh_radial_window(C.byref(S), events, ne, self._window_ws.data_ptr(),
                                        self._window_ws.numel(), sp), "lh_radial_window")
        host = out.cpu().numpy()
        return (host[:4 * cells].view(np.int32).reshape(ne, nb, n),
                host[4 * cells:8 * cells].view(np.int32).reshape(ne, nb, n),
                host[8 * cells:].view(np.float64).reshape(ne, nb, n))

    def attenuation(self, distance):
        radius, log_factor = self._attenuation
        return np.exp(np.interp(distance, radius, log_factor))

    def om_geometry(self, el, group_index, *, want_distance=True, want_earliest=False):
        """``min_distance_to_segments`` and ``earliest_element_arrival`` on the device."""
        import torch
        dev = self.device
        n = self.n_om
        t = {k: torch.tensor(np.ascontiguousarray(el[k], float), dtype=torch.float64, device=dev)
             for k in ("start_m", "direction", "length_m", "start_ns")}
        off = torch.tensor([0, len(el["length_m"])], dtype=torch.int64, device=dev)
        dist = torch.empty(n, dtype=torch.float64, device=dev) if want_distance else None
        early = torch.empty(n, dtype=torch.float64, device=dev) if want_earliest else None
        g = _lib.OmGeometry(n, self._pos.data_ptr(), 1, off.data_ptr(), t["start_m"].data_ptr(),
                            t["direction"].data_ptr(), t["length_m"].data_ptr(),
                            t["start_ns"].data_ptr(), float(group_index),
                            dist.data_ptr() if dist is not None else None,
                            early.data_ptr() if early is not None else None)
        sp = _lib.stream_ptr(torch.cuda.current_stream(dev))
        _lib.check(_lib.load().lh_om_geometry(C.byref(g), sp), "lh_om_geometry")
        return (dist.cpu().numpy() if dist is not None else None,
                early.cpu().numpy() if early is not None else None)


def _concat_elements(events):
    offsets = np.zeros(len(events) + 1, np.int64)
    offsets[1:] = np.cumsum([len(e["length_m"]) for e in events])
    cat = {k: np.concatenate([np.asarray(e[k], float) for e in events])
           for k in ("start_m", "direction", "length_m", "start_ns")}
    return offsets, cat


def delay_groups(el, *, prompt_delay_ns, cell_ns, window_end_ns, group_index_max):
    """``delay_groups`` (``shower/ge2.py:122-147``): steps split by their delay
    behind the light front of the earliest step. Prompt steps (delay <=
    ``prompt_delay_ns``) keep the source's clock; later steps are grouped in
    ``cell_ns`` cells, each shifted by its smallest delay, unless none of their
    light can arrive before the window ends (``beyond``: charge only).
    Returns ``(prompt_mask, [(mask, shift_ns)], beyond_mask)``."""
    start_ns = np.ascontiguousarray(el["start_ns"], float)
    start = np.ascontiguousarray(el["start_m"], float)
    first = int(np.argmin(start_ns))
    # (t - t_first) - |x - x_first| / c per step, one host pass of the library
    delay, distance = np.empty(len(start_ns)), np.empty(len(start_ns))
    _lib.check(_lib.load().lh_element_delays(len(start_ns), start.ctypes.data,
                                             start_ns.ctypes.data, first, C_M_PER_NS,
                                             delay.ctypes.data, distance.ctypes.data),
               "lh_element_delays")
    prompt = delay <= prompt_delay_ns
    beyond = ~prompt & (delay - (group_index_max - 1.0) * distance / C_M_PER_NS > window_end_ns)
    within = ~prompt & ~beyond
    groups = []
    if np.any(within):
        cells = np.floor(delay / cell_ns).astype(np.int64)
        for cell in np.unique(cells[within]):
            mask = within & (cells == cell)
            groups.append((mask, float(delay[mask].min())))
    return prompt, groups, beyond


def elements_of(source):
    """Element arrays of a shower source (reference objects or dicts with its names)."""
    el = getattr(source, "elements", source)
    if isinstance(el, ResidentElements):  # host arrays plus their device copies
        return el
    if isinstance(el, dict):
        out = {k: np.asarray(el[k], float) for k in ELEMENT_FIELDS}
        cone = el.get("cone_model", "spectral")
    else:
        out = {k: np.asarray(getattr(el, k), float) for k in ELEMENT_FIELDS}
        cone = getattr(el, "cone_model", "spectral")
    if cone != "spectral":
        raise ValueError("the shower route requires spectral cones (cone_model='spectral')")
    return out


def _subset(el, mask):
    return {k: v[mask] for k, v in el.items()}


class _Stages:
    """Wall time per route stage (``metadata['timings']``); with ``sync`` the
    device is synchronised at every boundary so each stage owns its GPU time."""

    def __init__(self, sync):
        self.sync = sync
        self.times = {}
        self.last = perf_counter()

    def __call__(self, name):
        if self.sync:
            import torch
            torch.cuda.synchronize()
        now = perf_counter()
        self.times[name] = self.times.get(name, 0.0) + now - self.last
        self.last = now


@dataclass
class _Lane:
    stream: object
    order1: object
    order1_screen: object
    source: object


@dataclass
class _Event:
    """Per-shower state carried between the stages of a batch."""
    el: dict
    extra: np.ndarray
    origins: np.ndarray | None = None
    frame: tuple = None
    reference: float = 0.0
    points: list = None
    coords: list = None
    channels: object = None
    zero_ch: list = None
    npts: np.ndarray = None
    used: np.ndarray = None
    tail: np.ndarray = None
    reach: np.ndarray = None
    predicted: np.ndarray = None
    local_origin: bool = False
    prompt_el: dict = None
    inside: np.ndarray = None
    work: np.ndarray = None
    charge: np.ndarray = None
    level1: np.ndarray = None
    bins1: np.ndarray = None
    fine: np.ndarray = None
    cone_cos: np.ndarray = None
    fused_el: dict = None       # elements of the fused order-1 unit (every band)
    fused_dev: dict = None      # their device arrays when they are all prompt elements
    fused_box: tuple = None
    units: list = field(default_factory=list)  # (band, elements) of the per-band units
    table: object = None
    pending: dict = field(default_factory=dict)


def settings_of(config, base=None):
    """``ShowerSettings`` from a reference ``ShowerConfig`` (``shower/api.py:47-90``:
    the predictor, delayed-light and screen fields the route reads), or the
    settings themselves."""
    from dataclasses import replace
    base = base or ShowerSettings()
    if config is None or isinstance(config, ShowerSettings):
        return config or base
    return replace(base, predictor_cell_m=float(config.predictor_cell_m),
                   predictor_safety=float(config.predictor_safety),
                   prompt_delay_ns=float(config.prompt_delay_ns),
                   delayed_cell_ns=float(config.delayed_cell_ns),
                   screen=bool(config.prompt.screen),
                   screen_margin=float(config.prompt.screen_margin),
                   min_distance_m=float(config.prompt.min_distance_m))


@functools.lru_cache(maxsize=1)
def response_class():
    """The reference's ``HybridTransportResponse`` when the reference package
    is importable (so that ``isinstance`` checks against it hold), else the
    local class with the same fields."""
    try:
        from lighthit.transport import HybridTransportResponse as Reference
    except ImportError:
        return HybridTransportResponse
    return Reference


class ShowerTransport:
    """``ShowerTransport(kernel, data=None, *, config=None, threads=None)(source, ...)``
    on the device route (``shower/api.py:114-318``).

    ``kernel`` is ``ShowerTables`` (the route's device tables) or the
    reference's ``TransportKernel``, whose prepared tables are then read once
    through the reference (``ShowerTables.from_reference`` with ``data``).
    ``config``: ``ShowerSettings`` or the reference's ``ShowerConfig``.
    ``threads`` is accepted for the reference's signature; the device route
    ignores it. ``batch(sources)`` runs many showers stage by stage: every stage
    launches its kernels for all showers back to back and the host reads the
    device once per stage, not once per shower. ``profile=True`` synchronises
    the device between stages so that ``metadata['timings']`` attributes the
    GPU time to each stage.
    """

    def __init__(self, kernel, data=None, *, config=None, threads=None, profile=False, lanes=4,
                 device="cuda"):
        if isinstance(kernel, ShowerTables):
            tables = kernel
        else:
            tables = ShowerTables.from_reference(kernel, data, config=config, device=device,
                                                 settings=settings_of(config))
        self.kernel = None if isinstance(kernel, ShowerTables) else kernel
        self.tables = tables
        self.config = settings_of(config, tables.settings)
        self.threads = threads
        self.profile = profile
        self.n_lanes = max(1, int(lanes))
        self._lane_list = None
        self._omega_dev = None

    # -- per-event launches on side streams -------------------------------------
    def _lanes(self):
        """Side streams for the per-event launch sequences of a batch (source
        compile, order-1 stages A and B), each with its own workspaces, so the
        small grids of several showers share the device."""
        import copy
        import torch
        if self._lane_list is None:
            T = self.tables
            lanes = []
            for _ in range(self.n_lanes):
                views = {}
                for name in ("order1", "order1_screen", "source"):
                    view = copy.copy(getattr(T, name))
                    view._workspace = None
                    view._pencil_pool = None
                    view._pool_table = None
                    view.__dict__.pop("_bands", None)  # per-band views own workspaces too
                    views[name] = view
                lanes.append(_Lane(torch.cuda.Stream(T.device), **views))
            self._lane_list = lanes
        return self._lane_list

    @contextmanager
    def _fan_out(self):
        """Lanes that start after the work queued so far on the current stream;
        on exit the current stream waits for all of them."""
        import torch
        main = torch.cuda.current_stream(self.tables.device)
        lanes = self._lanes()
        for lane in lanes:
            lane.stream.wait_stream(main)
        try:
            yield lanes
        finally:
            for lane in lanes:
                main.wait_stream(lane.stream)

    # -- order >=2 helpers ----------------------------------------------------
    def _apply_device(self, points, channels, reference, frame, oms, *, zero_frequency):
        """``apply_folded`` (``shower/ge2.py:99-119``) for the OMs ``oms``: device (OM, W)."""
        return self._apply_many([(points, channels, reference, frame, oms)],
                                zero_frequency=zero_frequency)[0]

    def _apply_many(self, requests, *, zero_frequency, mode="fp32"):
        """``_apply_device`` of several ``(points, channels, reference, frame, oms)``
        requests (the events of a batch) in one batched launch set per table."""
        T = self.tables
        out = [None] * len(requests)
        joint, split = [], []
        for i, (points, channels, reference, frame, oms) in enumerate(requests):
            centre, axis, first, second = frame
            basis = (centre, first, second, axis)
            args = (T.positions[oms], T.looks[oms], T.areas[oms], T.radial)
            if all(len(p) == len(points[0]) and np.array_equal(p, points[0]) for p in points[1:]):
                refs = np.broadcast_to(np.asarray(reference, float), (len(points),)).copy()
                src = AxialSources(points[0], channels, refs, basis, T.source_degree,
                                   T.azimuthal_degree)
                joint.append((i, (src,) + args))
            else:  # node bands with their own points: one band-view problem per band
                refs = np.broadcast_to(np.asarray(reference, float), (len(points),))
                for b in range(len(points)):
                    src = AxialSources(points[b], channels[b][None], refs[b:b + 1].copy(), basis,
                                       T.source_degree, T.azimuthal_degree)
                    split.append((i, b, (src,) + args))
        self.ge2_status = []  # status words of tensor-core contractions (read with the results)
        if joint:
            for (i, _), res in zip(joint, T.ge2.apply_batch([it for _, it in joint],
                                                            zero_frequency=zero_frequency,
                                                            mode=mode)):
                out[i] = res
            if T.ge2.status is not None:
                self.ge2_status.append(T.ge2.status)
        for b in sorted({b for _, b, _ in split}):
            part = [(i, it) for i, bb, it in split if bb == b]
            view = T.ge2.band(b)
            for (i, _), res in zip(part, view.apply_batch(
                    [it for _, it in part], zero_frequency=zero_frequency, mode=mode)):
                out[i] = res if out[i] is None else out[i] + res
            if view.status is not None:
                self.ge2_status.append(view.status)
        return out

    def __call__(self, source, *, progress=None, time_origin_ns=None,
                 selection_extra_charge=None, receivers=None):
        if receivers is not None:  # shower/api.py:205-212: those OMs, threshold zero
            return self._subset_route(receivers)(source, time_origin_ns=time_origin_ns,
                                                 selection_extra_charge=selection_extra_charge)
        return self.batch([source], time_origin_ns=None if time_origin_ns is None
                          else [time_origin_ns],
                          selection_extra_charge=None if selection_extra_charge is None
                          else [selection_extra_charge])[0]

    def _subset_route(self, receivers):
        """A route on ``tables.subset(receivers)`` (the last few kept: an event
        refines the same OM sets across its sources)."""
        key = tuple(int(v) for v in np.asarray(receivers, np.int64).ravel())
        cache = self.__dict__.setdefault("_subsets", {})
        if key not in cache:
            if len(cache) >= 8:
                cache.pop(next(iter(cache)))
            cache[key] = ShowerTransport(self.tables.subset(key), config=self.config,
                                         profile=self.profile, lanes=self.n_lanes)
        return cache[key]

    def batch(self, sources, *, time_origin_ns=None, selection_extra_charge=None):
        """Responses of several showers (``transport_shower`` per source)."""
        import torch
        began = perf_counter()
        stage = _Stages(self.profile)
        T, cfg = self.tables, self.config
        n = T.n_om
        omega, edges, threshold = T.omega, T.edges, T.threshold
        low, high = T.radial
        dev = T.device
        safety = float(cfg.predictor_safety)
        nb_bands = len(T.fold_bands)
        max_phase = float(np.max(T.phase))
        fastest = float(np.min(T.group))
        events = []
        # ---- per shower: elements, delay groups, frame (host)
        for k, source in enumerate(sources):
            el = elements_of(source)
            valid = el["beta"] * max_phase > 1
            if not np.any(valid):
                raise ValueError("source is below Cherenkov threshold over the wavelength range")
            if not np.all(valid):
                el = _subset(el, valid)
            given = None if selection_extra_charge is None else selection_extra_charge[k]
            extra = np.zeros(n) if given is None else np.maximum(np.asarray(given, float), 0.0)
            if extra.shape != (n,) or not np.isfinite(extra).all():
                raise ValueError("selection_extra_charge must hold one finite value per OM")
            prompt, late_groups, beyond = delay_groups(
                el, prompt_delay_ns=float(cfg.prompt_delay_ns), cell_ns=float(cfg.delayed_cell_ns),
                window_end_ns=float(edges[-1]), group_index_max=float(np.max(T.group)))
            ev = _Event(el, extra)
            # the order >=2 source of the prompt steps (orders 0 and 1 take every step)
            ev.src_el = el if np.all(prompt) else _subset(el, prompt)
            ev.late = None
            if not np.all(prompt):  # delayed light (shower/api.py:294-310)
                ev.late = {"zero_el": _subset(el, ~prompt),
                           "group_el": [(_subset(el, m), shift) for m, shift in late_groups],
                           "steps_in_groups": int(sum(int(m.sum()) for m, _ in late_groups)),
                           "beyond": int(beyond.sum())}
            src = ev.src_el
            ev.frame = axis_frame(src["start_m"], src["direction"], src["length_m"],
                                  src["coefficient0"])
            events.append(ev)
        store = ElementBatch([ev.el for ev in events], dev)  # one upload for every stage
        stage("setup")
        # the batch's status words, one zeroed allocation: the source compile's,
        # the prompt stages', then a screen and a fine word per shower
        words = torch.zeros(2 + 2 * len(events), dtype=torch.int32, device=dev)
        for k, ev in enumerate(events):
            ev.words = (words[2 + 2 * k:3 + 2 * k], words[3 + 2 * k:4 + 2 * k])
        # ---- order >=2 sources on the node bands (device, all showers)
        src_status = words[0:1]
        compiled = []
        with self._fan_out() as lanes:
            for k, ev in enumerate(events):
                lane = lanes[k % len(lanes)]
                with torch.cuda.stream(lane.stream):
                    compiled.append(lane.source.compile(
                        ev.src_el, ev.frame, status=src_status,
                        device_elements=store.event(k) if ev.src_el is ev.el else None))
        # one read of every shower's point counts, points and zero-frequency
        # channels (full capacity; sliced here) and the overflow flag
        host = _lib.fetch([src_status] + [t for c in compiled
                                          for t in (c[2], c[0], c[1][:, :, :, 0])])
        if int(host[0][0]) & _lib.LH_STATUS_OVERFLOW:
            raise ValueError("element nodes fall outside the source lattice")
        for k, (ev, c) in enumerate(zip(events, compiled)):
            npts, pts, zero = host[1 + 3 * k], host[2 + 3 * k], host[3 + 3 * k]
            _, ch_d, _, ev.reference, ev.frame = c
            ev.npts = npts
            centre, axis, e1, e2 = (np.asarray(v, float) for v in ev.frame)
            ev.coords = [p[:npts[b]] for b, p in enumerate(pts)]  # (z, x, y) in the frame
            ev.points = [centre + p[:npts[b], :1] * axis + p[:npts[b], 1:2] * e1
                         + p[:npts[b], 2:3] * e2 for b, p in enumerate(pts)]
            ev.channels = (ch_d[:, :int(npts[0])] if np.all(npts == npts[0])
                           else [ch_d[b, :int(npts[b])] for b in range(nb_bands)])
            ev.zero_ch = [zero[b, :int(npts[b])] for b in range(nb_bands)]
        for ev in events:  # delayed parts: their own frames and lattices (rare)
            if ev.late is None:
                continue
            ev.late["zero"] = self._part(T.source, ev.late["zero_el"])
            ev.late["groups"] = [(self._part(T.source, part), shift)
                                 for part, shift in ev.late["group_el"]]
        stage("source_compile")
        # ---- radial windows (shower/api.py:322-340, shower_basis.py:408-439)
        weight_ratio = float(np.sum(T.fold_scale) / np.sum(T.fold_scale[T.fold_bands]))
        window = [(c[0], c[1], ev.npts, ev.frame) for c, ev in zip(compiled, events)]
        owner = list(range(len(events)))
        for k, ev in enumerate(events):  # delayed steps' points count too (api.py:327-338)
            if ev.late is not None:
                z = ev.late["zero"]
                window.append((z["raw_points"], z["raw_channels"], z["npts"], z["frame"]))
                owner.append(k)
        n_near, n_far, far_sum = T.radial_window(window)
        acc = [(np.zeros(n, np.int64), np.zeros(n), np.zeros(n, bool)) for _ in events]
        for row, k in enumerate(owner):
            used, tail, near = acc[k]
            npts = window[row][2]
            for b, band in enumerate(T.fold_bands):
                used = np.maximum(used, int(npts[b]) - n_near[row, b] - n_far[row, b])
                tail = tail + weight_ratio * (10 * T.areas * T.peak_acceptance
                                              * T.efficiency[band] * far_sum[row, b])
            acc[k] = (used, tail, near | np.any(n_near[row] > 0, axis=0))
        for k, ev in enumerate(events):
            used, tail, near = acc[k]
            ev.near = bool(np.any(near))
            if ev.near and T.near is None:
                raise NotImplementedError("basis points inside the table's inner radius need the "
                                          "near-field table (tables/near_<config>.npz)")
            ev.used, ev.tail, ev.reach = used, tail, np.flatnonzero(used > 0)
        stage("radial_window")
        # ---- predictor (shower/ge2.py:70-96) and its zero-frequency charge (device)
        predict = []
        for ev in events:
            ev.predicted = np.zeros(n)
            if not len(ev.reach):
                continue
            centre, axis, e1, e2 = (np.asarray(v, float) for v in ev.frame)
            c_points, c_channels = [], []
            for b in range(nb_bands):
                # frame coordinates as compiled (a world round trip would move points
                # on the axis off 0 and across a predictor cell edge)
                coords = ev.coords[b]
                keys = np.floor(coords / float(cfg.predictor_cell_m)).astype(np.int64)
                keys -= keys.min(axis=0)
                span = keys.max(axis=0) + 1
                flat = (keys[:, 0] * span[1] + keys[:, 1]) * span[2] + keys[:, 2]
                _, inverse = np.unique(flat, return_inverse=True)
                groups = int(inverse.max()) + 1
                wgt = np.abs(ev.zero_ch[b][:, 0])
                total = np.bincount(inverse, weights=wgt, minlength=groups)
                count = np.bincount(inverse, minlength=groups)
                share = np.where(total[inverse] > 0,
                                 wgt / np.where(total > 0, total, 1.0)[inverse],
                                 1.0 / count[inverse])
                centroid = np.stack([np.bincount(inverse, weights=share * coords[:, k],
                                                 minlength=groups) for k in range(3)], axis=1)
                order = np.argsort(inverse, kind="stable")  # group sums in point order
                starts = np.searchsorted(inverse[order], np.arange(groups))
                summed = np.add.reduceat(ev.zero_ch[b][order].astype(complex), starts, axis=0)
                c_points.append(centre + centroid[:, :1] * axis + centroid[:, 1:2] * e1
                                + centroid[:, 2:3] * e2)
                c_channels.append(summed[:, :, None])
            c_ch = (np.stack(c_channels) if all(len(p) == len(c_points[0]) for p in c_points[1:])
                    else c_channels)
            ev.predictor_points = len(c_points[0])
            predict.append((ev, (c_points, c_ch, ev.reference, ev.frame, ev.reach)))
        for (ev, _), res in zip(predict, self._apply_many([r for _, r in predict],
                                                          zero_frequency=True)):
            ev.pending["predicted"] = res
        # ---- clocks (shower/api.py:455-477) and module selection distances (device)
        time_width = float(np.ptp(edges))
        for k, ev in enumerate(events):
            el = ev.el
            span = float(np.max(el["end_ns"]) - np.min(el["start_ns"]))
            # midpoints lie inside the box of starts and ends: the exact extent is
            # needed only when the box's extent passes the radial limit
            low_box, high_box = ev.box = element_box(el)
            extent = float(np.linalg.norm(high_box - low_box))
            if extent > high:
                mid = el["start_m"] + 0.5 * el["length_m"][:, None] * el["direction"]
                extent = float(np.linalg.norm([np.ptp(mid[:, k]) for k in range(3)]))
            ev.local_origin = extent > high or span > 0.5 * time_width
            given = None if time_origin_ns is None else time_origin_ns[k]
            if given is not None:
                ev.origins = np.asarray(given, float)
                if ev.origins.shape != (n,) or not np.isfinite(ev.origins).all():
                    raise ValueError("time_origin_ns must hold one finite origin per OM")
            elif not ev.local_origin:
                first = int(np.argmin(el["start_ns"]))
                ev.origins = (float(el["start_ns"][first])
                              + np.linalg.norm(T.positions - el["start_m"][first], axis=1)
                              / (C_M_PER_NS / fastest))
            pel = el
            pvalid = el["beta"] * T.threshold_phase > 1
            if not np.any(pvalid):
                raise ValueError("source is below Cherenkov threshold over the wavelength range")
            if not np.all(pvalid):
                pel = _subset(el, pvalid)
            ev.prompt_el = pel
            ev.prompt_box = ev.box if pel is el else element_box(pel)
        same = all(ev.prompt_el is ev.el for ev in events)
        prompt_store = store if same else ElementBatch([ev.prompt_el for ev in events], dev)
        dist_d, early_d = T.om_geometry_batch(prompt_store, store, fastest, host=False)
        pred = [ev for ev in events if "predicted" in ev.pending]
        host = _lib.fetch([dist_d, early_d] + [ev.pending.pop("predicted")[:, 0] for ev in pred])
        dist, early = host[0], host[1]
        for ev, values in zip(pred, host[2:]):
            ev.predicted[ev.reach] = values.real
        for k, ev in enumerate(events):
            if ev.origins is None:
                ev.origins = early[k]
        # delayed light is small and compact: its zero-frequency charge exactly on
        # every reachable OM (shower/api.py:345-352)
        late_req = [ev for ev in events if ev.late is not None and len(ev.reach)]
        for ev in events:
            ev.late_charge = np.zeros(n)
        if late_req:
            zs = [ev.late["zero"] for ev in late_req]
            for ev, res in zip(late_req, self._apply_many(
                    [(z["points"], self._zero_only(z["channels"]), z["reference"], z["frame"],
                      ev.reach) for z in zs], zero_frequency=True)):
                ev.late_charge[ev.reach] = res.cpu().numpy()[:, 0].real
        stage("predictor_clock")
        # ---- prompt orders 0 and 1 (transport_prompt, prompt.py:500-947)
        for k, ev in enumerate(events):
            self._prompt_selection(ev, dist[k], safety)
        prompt_events = [ev for ev in events if len(ev.work)]
        for k, ev in enumerate(events):
            ev.device_el = prompt_store.event(k)
        status = words[1:2]
        cone = float(np.sum(T.prompt["s0w"] * T.phase) / np.sum(T.prompt["s0w"]))
        for ev in prompt_events:
            self._order1_units(ev, cone)
            ev.status = ev.words[0]
        # the coarse order-1 screens run on the lanes while order 0 (one launch for
        # every shower) runs on this stream
        with self._fan_out() as lanes:
            if cfg.screen and threshold > 0:
                for k, ev in enumerate(prompt_events):
                    lane = lanes[k % len(lanes)]
                    with torch.cuda.stream(lane.stream):
                        if ev.fused_el is None:
                            ev.pending["coarse"] = torch.zeros(n, dtype=torch.float64,
                                                               device=dev)
                            continue
                        coarse = pencils(lane.order1_screen, ev.fused_el, ev.cone_cos,
                                         status=ev.status, device_elements=ev.fused_dev,
                                         box=ev.fused_box)
                        ev.pending["coarse"] = grouped(lane.order1_screen, coarse, ev.work,
                                                       ev.origins, status=ev.status)[0]
            if prompt_events:
                origins = np.stack([ev.origins for ev in prompt_events])
                batch0 = (prompt_store if len(prompt_events) == len(events) else
                          ElementBatch([ev.prompt_el for ev in prompt_events], dev))
                out0 = order0(T.order0, batch0, origins, edges, check=False,
                              estimate=cfg.order0_check > 0)
        if prompt_events:
            extra0 = [out0["status"], out0["charge"]]
            if out0["charge_check"] is not None:
                extra0.append(out0["charge_check"])
            coarse_host = self._collect(prompt_events, "coarse", T.order1_screen, extra0)
            raise_order0_status(int(extra0[0][0]))
            q0_all = extra0[1]
            bins0_all = out0["bins"]
            for k, ev in enumerate(prompt_events):
                ev.charge[ev.work, 0] = q0_all[k][ev.work]
                ev.pending["bins0"] = bins0_all[k]
                if len(extra0) > 2:
                    q = q0_all[k][ev.work]
                    failed = ev.work[np.abs(q - extra0[2][k][ev.work])
                                     > self._order0_tolerance(q, 1.0)]
                    if len(failed):
                        self._order0_converged(ev, failed, bins0_all[k])
        stage("order0_screen")
        fine_events = []
        for ev in prompt_events:
            ev.fine = ev.work
            if id(ev) in coarse_host:
                coarse = coarse_host[id(ev)]
                if ev.units:
                    coarse = coarse + self._units_charge(ev, ev.work, coarse=True)[0]
                ev.charge[ev.work, 1] = coarse[ev.work]
                ev.level1[ev.work] = 1
                ev.pending["coarse_host"] = coarse
                ev.fine = ev.work[(ev.charge[ev.work, 0] + ev.extra_prompt[ev.work]
                                   + cfg.screen_margin * np.maximum(coarse[ev.work], 0.0))
                                  >= threshold]
            if len(ev.fine):
                ev.status = ev.words[1]
                fine_events.append(ev)
        with self._fan_out() as lanes:
            for k, ev in enumerate(fine_events):
                lane = lanes[k % len(lanes)]
                with torch.cuda.stream(lane.stream):
                    if ev.fused_el is None:
                        ev.pending["fine"] = (
                            torch.zeros(n, dtype=torch.float64, device=dev),
                            torch.zeros((n, len(edges) - 1), dtype=torch.float64, device=dev))
                        continue
                    ev.table = pencils(lane.order1, ev.fused_el, ev.cone_cos, status=ev.status,
                                       device_elements=ev.fused_dev, box=ev.fused_box)
                    ev.pending["fine"] = grouped(lane.order1, ev.table, ev.fine, ev.origins,
                                                 status=ev.status)
        fine_host = self._collect(prompt_events, "fine", T.order1)
        for ev in prompt_events:
            if id(ev) not in fine_host:
                continue
            q1, b1 = fine_host[id(ev)]
            if ev.units:
                qu, bu = self._units_charge(ev, ev.fine)
                q1, b1 = q1 + qu, b1 + bu
            ev.charge[ev.fine, 1] = q1[ev.fine]
            ev.bins1[ev.fine] = b1[ev.fine]
            ev.level1[ev.fine] = 2
            coarse = ev.pending.pop("coarse_host", None)
            if coarse is not None:  # widening (prompt.py:776-805)
                worst = float(np.min(coarse[ev.fine] / np.maximum(q1[ev.fine], 1e-300)))
                if worst * cfg.screen_margin < 1.0:
                    wider = 1.5 / max(worst, 1e-3)
                    more = ev.work[(ev.level1[ev.work] == 1)
                                   & (ev.charge[ev.work, 0] + ev.extra_prompt[ev.work] + wider
                                      * np.maximum(coarse[ev.work], 0.0) >= threshold)]
                    if len(more):
                        q1m, b1m = self._fine_order1(ev, more, status)
                        ev.charge[more, 1] = q1m[more]
                        ev.bins1[more] = b1m[more]
                        ev.level1[more] = 2
        stage("order1")
        # ---- exact zero-frequency >=2 where the decision needs it (shower/api.py:488-525)
        exact_req = []
        for ev in events:
            ev.pending["ge2"] = {}
            prompt_charge = ev.charge.sum(axis=1)
            ev.computable = (ev.used > 0) | (prompt_charge > 0)
            cand = (ev.used > 0) & (prompt_charge + safety * np.abs(ev.predicted)
                                    + ev.late_charge + ev.extra >= threshold)
            if threshold == 0:
                cand = ev.used > 0
            ev.candidate = cand
            ids = np.flatnonzero(cand)
            if len(ids):
                exact_req.append((ev, ids))
        exact_res = self._apply_many(
            [(ev.points, self._zero_only(ev.channels), ev.reference, ev.frame, ids)
             for ev, ids in exact_req], zero_frequency=True)
        # one read: the order-1 status word and every exact charge
        host = _lib.fetch([status] + [res[:, 0] for res in exact_res])
        if int(host[0][0]) & _lib.LH_STATUS_OVERFLOW:
            raise MemoryError("order-1 tables overflowed their device capacity")
        for (ev, ids), values in zip(exact_req, host[1:]):
            ev.pending["exact"] = (ids, values)
        for ev in events:
            exact = np.zeros(n)
            if "exact" in ev.pending:
                ids, values = ev.pending.pop("exact")
                exact[ids] = values.real
            cand = ev.candidate
            ratio = np.abs(exact[cand]) / np.maximum(np.abs(ev.predicted[cand]), 1e-300)
            fallback = bool(np.any(np.abs(exact[cand]) > safety * np.abs(ev.predicted[cand])))
            if fallback:  # the prediction failed its own margin: every reachable OM exact
                cand = ev.used > 0
                ids = np.flatnonzero(cand)
                exact = np.zeros(n)
                if len(ids):
                    exact[ids] = self._apply_device(ev.points, self._zero_only(ev.channels),
                                                    ev.reference, ev.frame, ids,
                                                    zero_frequency=True).cpu().numpy()[:, 0].real
            ev.fallback, ev.ratio, ev.candidate = fallback, ratio, cand
            charge2 = ev.predicted + ev.late_charge
            charge2[cand] = exact[cand] + ev.late_charge[cand]
            ev.charge = np.column_stack((ev.charge, charge2))
            level = np.where(ev.used > 0, 1, 0).astype(np.int8)
            level[cand] = 2
            ev.level2 = level
            active = ev.computable & (ev.charge.sum(axis=1) + ev.extra >= threshold)
            if threshold == 0:
                active = ev.computable
            if np.any(active & (level == 1)):
                raise RuntimeError("an OM was activated by a predicted >=2 charge")
            ev.active = active
        stage("ge2_exact_zero")
        # ---- full frequencies for the active OMs, the prompt bins they lack, the readout
        row_ev = []
        for k, ev in enumerate(events):
            ev.spectrum = np.zeros((len(omega), n), complex)
            ids = np.flatnonzero(ev.active)
            missing = np.flatnonzero(ev.active & (ev.level1 < 2))
            if len(missing):  # the reference reruns the prompt without its screen
                q1m, b1m = self._fine_order1(ev, missing, status)
                ev.charge[missing, 1] = q1m[missing]
                ev.bins1[missing] = b1m[missing]
            work = np.flatnonzero(ev.active & (ev.used > 0))
            if len(work):
                row_ev.append((k, work))
        if row_ev:
            specs = self._apply_many([(events[k].points, events[k].channels, events[k].reference,
                                       events[k].frame, work) for k, work in row_ev],
                                     zero_frequency=False, mode=cfg.contraction_mode)
            contraction_status = list(self.ge2_status)
            # relative-time spectra e^{-i w origin} N(w); the stored zero frequency is
            # the exact >=2 charge (shower/api.py:584)
            origin = np.concatenate([events[k].origins[work] for k, work in row_ev])
            zero = np.concatenate([events[k].charge[work, 2] - events[k].late_charge[work]
                                   for k, work in row_ev])
            # the phases e^{-i w origin} on the device (one upload of the origins
            # and zero-frequency charges)
            packed = _lib.upload(np.concatenate([origin, zero]), torch.float64, dev)
            rows = len(origin)
            if getattr(self, "_omega_dev", None) is None:
                self._omega_dev = torch.tensor(omega, dtype=torch.float64, device=dev)
            angle = torch.outer(packed[:rows], self._omega_dev).neg_()
            rel = torch.cat(specs) * torch.polar(torch.ones_like(angle), angle)
            rel[:, 0] = packed[rows:]
            bins2_d, _ = T.readout.bins(rel.to(torch.complex64), mode=cfg.readout_mode)
        # one read: the >=2 bins and spectra of the active OMs, the order-0 bins
        with_bins0 = [k for k, ev in enumerate(events) if np.any(ev.active)]
        host = _lib.fetch(([bins2_d] + list(specs) if row_ev else [])
                          + [events[k].pending["bins0"] for k in with_bins0]
                          + (contraction_status if row_ev else []))
        if row_ev and any(int(st[0]) & _lib.LH_STATUS_TIMEOUT
                          for st in host[len(host) - len(contraction_status):]):
            raise RuntimeError("the tensor-core >=2 contraction timed out waiting for its "
                               "pipeline")
        if row_ev:
            bins2 = host[0].astype(float)
            for (k, work), spec in zip(row_ev, host[1:1 + len(row_ev)]):
                events[k].pending["spec"] = (work, spec)
        for k, values in zip(with_bins0, host[(1 + len(row_ev)) if row_ev else 0:]):
            override = getattr(events[k], "order0_override", None)
            if override is not None:  # OMs whose order 0 was evaluated again
                values = np.array(values)
                values[override[0]] = override[1]
            events[k].pending["bins0"] = values
        late_bins = self._late_bins(events, row_ev, omega, cfg.readout_mode)
        responses = []
        row = 0
        row_map = {k: work for k, work in row_ev}
        for k, ev in enumerate(events):
            if "spec" in ev.pending:
                work, spec = ev.pending.pop("spec")
                ev.spectrum[:, work] = spec.T
            ev.spectrum[0] = ev.charge[:, 2] - ev.late_charge  # prompt steps (api.py:450)
            components = np.zeros((n, len(edges) - 1, 3))
            ids = np.flatnonzero(ev.active)
            if len(ids):
                if not np.all(ev.inside[ids]):
                    raise ValueError("prompt did not compute every active OM")
                components[ids, :, 0] = ev.pending["bins0"][ids]
                components[ids, :, 1] = ev.bins1[ids]
                if k in row_map:
                    work = row_map[k]
                    components[work, :, 2] = bins2[row:row + len(work)]
                    row += len(work)
                    for values in late_bins.get(k, []):
                        components[work, :, 2] += values
            metadata = {
                "route": "lighthit_b200.shower", "ge2_charge_level": ev.level2.tolist(),
                "ge2_predictor": {"points": int(getattr(ev, "predictor_points", 0)),
                                  "cell_m": float(cfg.predictor_cell_m), "safety": safety,
                                  "candidates": int(ev.candidate.sum()),
                                  "reachable": int(len(ev.reach)),
                                  "fallback_to_exact": ev.fallback,
                                  "exact_over_prediction_max": float(ev.ratio.max(initial=0.0)),
                                  "exact_over_prediction_min": (float(ev.ratio.min())
                                                                if len(ev.ratio) else None)},
                "prompt_order1_level": ev.level1.tolist(), "radial_window_m": [low, high],
                "order0": {"gauss_order": int(cfg.order0_gauss),
                           "check_order": int(cfg.order0_check),
                           "reevaluated_oms": (len(ev.order0_override[0])
                                               if getattr(ev, "order0_override", None)
                                               else 0),
                           "highest_order": int(getattr(ev, "order0_orders",
                                                        cfg.order0_gauss))},
                "radial_tail_estimate_max_pe": float(ev.tail.max(initial=0.0)),
                "time_origin": ("supplied event clock" if time_origin_ns is not None else
                                "earliest local segment and fastest group flight"
                                if ev.local_origin
                                else "earliest element start and fastest group flight"),
                "active_modules": int(ev.active.sum()), "threshold_pe": threshold,
                "ge2_points": [int(v) for v in ev.npts], "source_elements": len(ev.el["beta"]),
                "elapsed_seconds": (perf_counter() - began) / len(events),
                "batch_size": len(events), "timings": stage.times,
                "delayed_light": {
                    "prompt_delay_ns": float(cfg.prompt_delay_ns),
                    "delayed_cell_ns": float(cfg.delayed_cell_ns),
                    "groups_in_window": 0 if ev.late is None else len(ev.late["groups"]),
                    "steps_in_window_groups": 0 if ev.late is None else ev.late["steps_in_groups"],
                    "steps_beyond_window": 0 if ev.late is None else ev.late["beyond"],
                    "delayed_charge_pe": float(ev.late_charge.sum()),
                    "stored_spectrum": "prompt steps only (delayed light in charge and bins)"}}
            response = response_class()(
                None if self.kernel is None else self.kernel.detector, omega.copy(),
                edges.copy(), ev.spectrum, components, ev.charge, ev.origins, ev.active,
                "shower", metadata)
            if ev.near:  # shower/api.py:536-538
                origins = _lib.upload(ev.origins, torch.float64, dev)
                near = T.near.field(store.event(k), len(ev.el["beta"]), T._pos, T._looks,
                                    T._areas, origins)
                add_near_field(response, near, T.readout, mode=cfg.readout_mode, label="shower")
            responses.append(response)
        stage("ge2_full_readout")
        return responses

    def _part(self, compiler, part):
        """Source compile of a delayed part with its own frame: world points per
        band, device channels, host zero-frequency channels, sizes, frame."""
        frame = axis_frame(part["start_m"], part["direction"], part["length_m"],
                           part["coefficient0"])
        pts_d, ch_d, npts_d, reference, frame = compiler.compile(part, frame)
        npts = npts_d.cpu().numpy()
        pts = pts_d.cpu().numpy()
        centre, axis, e1, e2 = (np.asarray(v, float) for v in frame)
        nb = len(npts)
        return {"points": [centre + pts[b, :npts[b], :1] * axis + pts[b, :npts[b], 1:2] * e1
                           + pts[b, :npts[b], 2:3] * e2 for b in range(nb)],
                "channels": (ch_d[:, :int(npts[0])] if np.all(npts == npts[0])
                             else [ch_d[b, :int(npts[b])] for b in range(nb)]),
                "npts": npts, "reference": reference, "frame": frame,
                "raw_points": pts_d, "raw_channels": ch_d}

    def _late_bins(self, events, row_ev, omega, mode):
        """Bins of the delayed groups for the readout OMs: each group's spectrum
        demodulated by its own delay and read on the window edges seen from
        it (shower/api.py:466-477). ``{event: [bins per group]}``."""
        import torch
        T = self.tables
        req, meta = [], []
        for k, work in row_ev:
            ev = events[k]
            if ev.late is None:
                continue
            for g, shift in ev.late["groups"]:
                req.append((g["points"], g["channels"], g["reference"], g["frame"], work))
                meta.append((k, work, shift))
        out = {}
        if not req:
            return out
        for (k, work, shift), spec in zip(meta, self._apply_many(req, zero_frequency=False)):
            phase = _lib.upload(np.exp(-1j * np.outer(events[k].origins[work] + shift, omega)),
                                torch.complex128, T.device)
            values, _ = T.readout_shifted(shift).bins((spec * phase).to(torch.complex64),
                                                      mode=mode)
            out.setdefault(k, []).append(values.cpu().numpy().astype(float))
        return out

    def _order0_tolerance(self, q, fraction):
        """Allowed change of order-0 charges ``q`` between two quadrature orders:
        ``fraction`` of the reference's tolerance (``BallisticInterval.tolerance``,
        ``_surface_ballistic.py:88-89``), at least the float32 floor."""
        cfg = self.config
        reference = fraction * (cfg.order0_absolute_tolerance_pe
                                + cfg.order0_relative_tolerance * np.abs(q))
        return np.maximum(reference, cfg.order0_float32_floor * np.abs(q))

    def _order0_converged(self, ev, oms, bins_device):
        """Order 0 of the OMs ``oms`` whose error estimate failed: the Gauss order
        doubled from the route's until successive charges agree within a
        quarter of the reference's tolerance or the float32 floor (the
        ``adaptive`` loop of ``_surface_ballistic.py:179-196``, its ``rays``
        part); the reference's ``ValueError`` when the maximum order does not
        converge. The bins of the last order are kept. Unlike the reference's
        loop the bins' L1 change is not tested: node positions decide which bin
        each float32 sample lands in, so successive orders move ~1e-4 of an
        OM's charge between neighbouring bins (measured on the README shower
        and the config-2 stream: 4e-4 from order 6 to 12, 4e-6 from 48 to
        64), inside the route's 1e-3 bins tolerance but far above the
        reference's 5e-7. Sets the charges on the event and keeps the bins
        for the final read."""
        import torch
        T, cfg = self.tables, self.config
        dev = T.device
        nb = len(T.edges) - 1
        prev_q = ev.charge[oms, 0].copy()
        ids_t = torch.as_tensor(oms, device=dev)
        prev_b = _lib.fetch([bins_device.index_select(0, ids_t)])[0]
        q_out, b_out = prev_q.copy(), prev_b.copy()
        pending = np.arange(len(oms))
        order = int(cfg.order0_gauss)
        elements = ElementBatch([ev.prompt_el], dev)
        while len(pending):
            order = min(2 * order, int(cfg.order0_max_order))
            optics = T.order0.subset(oms[pending], order=order)
            out = order0(optics, elements, ev.origins[oms[pending]][None], T.edges, check=False)
            status, q, b = _lib.fetch([out["status"], out["charge"][0], out["bins"][0]])
            raise_order0_status(int(status[0]))
            error = np.abs(q - prev_q[pending])
            bad = error > self._order0_tolerance(q, 0.25)
            q_out[pending], b_out[pending] = q, b
            if bad.any() and order == int(cfg.order0_max_order):
                worst = float(np.max(error[bad] / np.maximum(np.abs(q[bad]), 1e-300)))
                raise ValueError(f"ballistic rays quadrature failed for {int(bad.sum())} OMs "
                                 f"at order {order} (largest change {worst:.2e} of the charge)")
            prev_q[pending], prev_b[pending] = q, b
            pending = pending[bad]
        ev.charge[oms, 0] = q_out
        ev.order0_override = (np.asarray(oms), b_out.reshape(len(oms), nb))
        ev.order0_orders = order

    def _collect(self, events, key, tables, extra=None):
        """Host values of the events' pending ``key`` results (coarse charge, or
        fine charge and bins) read in one wait with their status words and the
        tensors of ``extra`` (replaced in place by their host arrays). Events
        whose bounded pencil table overflowed run stage A and B again at full
        size. Returns ``{id(event): host values}``."""
        pend = [ev for ev in events if key in ev.pending]
        extra = [] if extra is None else extra
        parts = list(extra) + [ev.status for ev in pend]
        for ev in pend:
            parts.extend([ev.pending[key]] if key == "coarse" else list(ev.pending[key]))
        host = _lib.fetch(parts) if parts else []
        extra[:] = host[:len(extra)]
        flags = host[len(extra):len(extra) + len(pend)]
        values = host[len(extra) + len(pend):]
        out = {}
        width = 1 if key == "coarse" else 2
        for i, (ev, f) in enumerate(zip(pend, flags)):
            got = values[width * i:width * (i + 1)]
            ev.pending.pop(key)
            if f[0] & _lib.LH_STATUS_OVERFLOW:
                table = pencils(tables, ev.fused_el, ev.cone_cos, device_elements=ev.fused_dev,
                                capacity_full=True, box=ev.fused_box)
                work = ev.work if key == "coarse" else ev.fine
                res = grouped_widening(tables, table, work, ev.origins)
                got = _lib.fetch([res[0]] if key == "coarse" else list(res))
                if key == "fine":
                    ev.table = table
            out[id(ev)] = got[0] if key == "coarse" else tuple(got)
        return out

    def _order1_units(self, ev, cone):
        """Order-1 evaluation units (``prompt.py:683-719`` with
        ``muon/secondary_first.py:184-204``): one fused unit of the elements
        above the Cherenkov threshold in every band (shared pencils, one cone at
        the s0w-weighted mean phase index) and, per band, a unit of the elements
        emitting in that band but not in all of them (that band's tables and
        cone, the unfused pencil resolution)."""
        T = self.tables
        el = ev.prompt_el
        beta = el["beta"]
        everywhere = beta * float(np.min(T.phase)) > 1  # rounding is monotone in n
        ev.units = []
        if np.all(everywhere):
            ev.fused_el, ev.fused_dev, ev.fused_box = el, ev.device_el, ev.prompt_box
            ev.cone_cos = 1.0 / (ev.device_el["beta"] * cone)
            return
        for band, phase in enumerate(T.phase):
            mask = (beta * float(phase) > 1) & ~everywhere
            if np.any(mask):
                ev.units.append((band, _subset(el, mask)))
        ev.fused_el = _subset(el, everywhere) if np.any(everywhere) else None
        ev.fused_dev = None
        ev.fused_box = None if ev.fused_el is None else element_box(ev.fused_el)
        ev.cone_cos = None if ev.fused_el is None else 1.0 / (ev.fused_el["beta"] * cone)

    def _units_charge(self, ev, oms, *, coarse=False):
        """Order-1 charge (and bins) at ``oms`` of an event's per-band units, summed."""
        T = self.tables
        charge = np.zeros(T.n_om)
        bins = None if coarse else np.zeros((T.n_om, len(T.edges) - 1))
        for band, sub in ev.units:
            tables = T.order1_band(band, coarse=coarse)
            table = pencils(tables, sub, 1.0 / (sub["beta"] * float(T.phase[band])),
                            capacity_full=True)
            q, b = grouped_widening(tables, table, oms, ev.origins)
            charge[oms] += q.cpu().numpy()[oms]
            if bins is not None:
                bins[oms] += b.cpu().numpy()[oms]
        return charge, bins

    def _fine_order1(self, ev, oms, status):
        """Full-resolution order 1 at ``oms`` over every unit (host arrays)."""
        T = self.tables
        q = np.zeros(T.n_om)
        b = np.zeros((T.n_om, len(T.edges) - 1))
        if ev.fused_el is not None:
            table = pencils(T.order1, ev.fused_el, ev.cone_cos, status=status,
                            device_elements=ev.fused_dev, capacity_full=True, box=ev.fused_box)
            q1, b1 = grouped_widening(T.order1, table, oms, ev.origins)
            q, b = q1.cpu().numpy(), b1.cpu().numpy()
        if ev.units:
            qu, bu = self._units_charge(ev, oms)
            q, b = q + qu, b + bu
        return q, b

    @staticmethod
    def _zero_only(channels):
        return ([c[:, :, :1] for c in channels] if isinstance(channels, list)
                else channels[:, :, :, :1])

    def _prompt_selection(self, ev, distance, safety):
        """Module selection of ``transport_prompt`` (``prompt.py:603-631``)."""
        T, cfg = self.tables, self.config
        n = T.n_om
        threshold = T.threshold
        el = ev.prompt_el
        max_distance = T.radial[1]
        inside = distance <= max_distance
        s0 = 1.0 / T.wavelengths ** 2
        s2 = s0 / T.phase ** 2
        emitted = float(sum(T.weights[b] * np.maximum(el["coefficient0"] * s0[b]
                                                      + el["coefficient2"] * s2[b], 0.0).sum()
                            for b in range(len(s0))))
        far = np.maximum(distance, 1e-9)
        upper = (10 * max(emitted, 0.0) * T.areas * T.peak_acceptance * float(np.max(T.efficiency))
                 * np.exp(-float(np.min(T.absorption)) * far) / (4 * np.pi * far ** 2))
        unsafe = (~inside) & (upper >= threshold)
        if np.any(unsafe):
            raise ValueError(f"{int(unsafe.sum())} OMs beyond max_distance_m={max_distance:g} have "
                             "a conservative estimate above threshold; increase max_distance_m")
        too_close = inside & (distance < cfg.min_distance_m)
        if np.any(too_close):
            raise ValueError(f"{int(too_close.sum())} OMs are closer than min_distance_m="
                             f"{cfg.min_distance_m:g} m to the source")
        ev.inside = inside
        ev.work = np.flatnonzero(inside)
        ev.charge = np.zeros((n, 2))
        ev.level1 = np.zeros(n, np.int8)
        ev.bins1 = np.zeros((n, len(T.edges) - 1))
        ev.extra_prompt = safety * np.abs(ev.predicted) + np.abs(ev.late_charge) + ev.extra
        ev.pending["bins0"] = None


def main(argv=None):
    """Run the first showers of the seeded config-2 stream: ``python -m lighthit_b200.shower``."""
    import argparse
    import json
    import torch
    from .workloads import gaussian_shower, shower_stream
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--tables", default="c2", choices=["c0", "c2"])
    ap.add_argument("--showers", type=int, default=8)
    ap.add_argument("--profile", action="store_true", help="per-stage device-synchronised times")
    ap.add_argument("--batch", action="store_true",
                    help="route all showers as one stage-major batch")
    args = ap.parse_args(argv)
    route = ShowerTransport(ShowerTables.synthetic(args.tables), profile=args.profile)
    draws = shower_stream(args.showers, route.tables.positions.mean(axis=0))
    showers = [gaussian_shower(d["position_m"], d["direction"],
                               charged_track_length_m=d["charged_track_length_m"],
                               elements=d["elements"], seed=d["seed"]) for d in draws]
    if args.batch:
        began = perf_counter()
        responses = route.batch(showers)
        torch.cuda.synchronize()
        elapsed = perf_counter() - began
    else:
        responses = []
        for el in showers:
            responses.append(route(el))
            torch.cuda.synchronize()
    for d, r in zip(draws, responses):
        print(json.dumps({"elements": d["elements"], "active": int(r.active.sum()),
                          "charge_pe": float(r.charge_pe.sum()),
                          "ms": 1e3 * r.metadata["elapsed_seconds"]}), flush=True)
    if args.batch:
        print(json.dumps({"batch_showers": len(showers), "batch_ms": 1e3 * elapsed,
                          "showers_per_s": len(showers) / elapsed}), flush=True)


if __name__ == "__main__":
    main()
