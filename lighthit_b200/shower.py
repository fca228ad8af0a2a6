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
* clocks and module selection: ``lh_om_geometry`` (float64, bit-identical).

Tables are built once by the reference and stored under ``tables/``
(``build_tables.py``): the folded >=2 kernels and the route's medium and
detector constants. What the device route does not cover raises
``NotImplementedError`` with the reason (delayed light groups, basis points
inside the table's inner radius, elements below threshold in a node band).
Order 1 follows the reference's global screen (``prompt.py:720-812``): a
coarse charge pass (2 m cells, 8-pixel faces, 24 ring nodes) for every OM in
reach, full resolution where ``q0 + extra + 3 q1_coarse`` reaches threshold,
widened when the coarse pass underestimated. The coarse pass is the grouped
evaluator on coarse pencils; the reference refines its coarse pixels near each
OM (``_prompt_screen.py``), so coarse-only OMs (below threshold by
construction) carry a different coarse order-1 charge.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from pathlib import Path
from time import perf_counter

import numpy as np

from . import _lib
from .ge2 import AxialSources, Ge2Table
from .order0 import Order0Optics, order0
from .order1 import Order1Tables, PromptSettings, acceptance_monomials, grouped, pencils
from .readout import DeviceReadout
from .source import ShowerBasisSettings, SourceCompiler, axis_frame

__all__ = ["ShowerSettings", "ShowerTables", "ShowerTransport", "HybridTransportResponse"]

C_M_PER_NS = 0.299792458
TABLES = Path(__file__).resolve().parent / "tables"
ELEMENT_FIELDS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
                  "start_ns", "end_ns")


@dataclass(frozen=True)
class ShowerSettings:
    """``ShowerConfig`` fields the route reads (``shower/api.py:47-90``)."""
    predictor_cell_m: float = 2.0
    predictor_safety: float = 2.0
    prompt_delay_ns: float = 20.0
    min_distance_m: float = 0.1          # PromptConfig.min_distance_m
    readout_mode: str = "split-bf16"
    order0_gauss: int = 8
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

    def __init__(self, route, folded, *, device="cuda", settings=ShowerSettings()):
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
        optics = {k: np.asarray(r[f"optics_{k}"], float) for k in (
            "panel_edges", "phase_nodes", "group_nodes", "extinction_nodes",
            "efficiency_coefficients")}
        self.order0 = Order0Optics(optics, self.positions, self.looks, self.areas, self.radii,
                                   self.alpha, order=settings.order0_gauss, device=device)
        self.order1 = Order1Tables(self.prompt, self.g, acceptance_monomials(self.alpha),
                                   self.positions, self.looks, self.areas, self.edges,
                                   settings=PromptSettings(), device=device)
        self.order1_screen = Order1Tables(self.prompt, self.g, acceptance_monomials(self.alpha),
                                          self.positions, self.looks, self.areas, self.edges,
                                          settings=PromptSettings().screen(), compute_bins=False,
                                          device=device)
        bands = self.fold_bands
        self.source = SourceCompiler(self.wavelengths[bands], self.fold_phase,
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
        self._pos = torch.tensor(self.positions, dtype=torch.float64, device=self.device)
        # spectral_attenuation (shower_basis.py:388-405) for the far-tail screen
        w = self.weights * self.efficiency / self.wavelengths ** 2
        lowest = float(self.absorption.min())
        radius = np.geomspace(1e-3, 1e5, 1025)
        log_factor = (np.log(np.exp(-np.outer(radius, self.absorption - lowest)) @ w / w.sum())
                      - lowest * radius)
        self._attenuation = (radius, log_factor)
        self.n_om = n

    @classmethod
    def synthetic(cls, name="c0", **kw):
        """Synthetic Baikal-like workloads: ``c0`` (48 OMs, 2-150 m), ``c2`` (384 OMs, 2-450 m)."""
        folded = {"c0": "ge2_fold_48om_2-150m.npz", "c2": "ge2_fold_384om_2-450m.npz"}
        if name not in folded:
            raise ValueError("known synthetic tables: c0, c2")
        return cls(TABLES / f"route_{name}.npz", TABLES / folded[name], **kw)

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


def elements_of(source):
    """Element arrays of a shower source (reference objects or dicts with its names)."""
    el = getattr(source, "elements", source)
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


class ShowerTransport:
    """``ShowerTransport(kernel, data)(source, ...)`` on the device route.

    ``profile=True`` synchronises the device between stages so that
    ``metadata['timings']`` attributes the GPU time to each stage.
    """

    def __init__(self, tables: ShowerTables, config: ShowerSettings | None = None, *,
                 profile=False):
        self.tables = tables
        self.config = config or tables.settings
        self.profile = profile

    def _apply(self, points, channels, reference, frame, oms, *, zero_frequency):
        """``apply_folded`` (``shower/ge2.py:99-119``) for the OMs ``oms``: (frequency, OM)."""
        T = self.tables
        W = 1 if zero_frequency else len(T.omega)
        if not len(oms):
            return np.zeros((W, 0), complex)
        centre, axis, first, second = frame
        area = T.areas[oms]
        same = all(len(p) == len(points[0]) and np.array_equal(p, points[0]) for p in points[1:])
        if same:
            src = AxialSources(points[0], channels, np.full(len(points), reference),
                               (centre, first, second, axis), T.source_degree, T.azimuthal_degree)
            return T.ge2.apply(src, T.positions[oms], T.looks[oms], area, T.radial,
                               zero_frequency=zero_frequency)
        total = 0
        for b in range(len(points)):
            src = AxialSources(points[b], channels[b][None], np.array([reference]),
                               (centre, first, second, axis), T.source_degree, T.azimuthal_degree)
            total = total + T.ge2.band(b).apply(src, T.positions[oms], T.looks[oms], area,
                                                T.radial, zero_frequency=zero_frequency)
        return total

    def __call__(self, source, *, time_origin_ns=None, selection_extra_charge=None,
                 receivers=None):
        import torch
        if receivers is not None:
            raise NotImplementedError("receiver subsets: build ShowerTables for those OMs")
        began = perf_counter()
        stage = _Stages(self.profile)
        T, cfg = self.tables, self.config
        n = T.n_om
        omega, edges, threshold = T.omega, T.edges, T.threshold
        low, high = T.radial
        el = elements_of(source)
        max_phase = float(np.max(T.phase))
        valid = el["beta"] * max_phase > 1
        if not np.any(valid):
            raise ValueError("source is below Cherenkov threshold over the wavelength range")
        if not np.all(valid):
            el = _subset(el, valid)
        extra = (np.zeros(n) if selection_extra_charge is None
                 else np.maximum(np.asarray(selection_extra_charge, float), 0.0))
        if extra.shape != (n,) or not np.isfinite(extra).all():
            raise ValueError("selection_extra_charge must hold one finite value per OM")
        # delay groups (shower/ge2.py:122-147): the device route handles prompt steps
        first = int(np.argmin(el["start_ns"]))
        distance0 = np.linalg.norm(el["start_m"] - el["start_m"][first], axis=1)
        delay = el["start_ns"] - el["start_ns"][first] - distance0 / C_M_PER_NS
        if np.any(delay > cfg.prompt_delay_ns):
            raise NotImplementedError("delayed light groups (steps more than prompt_delay_ns "
                                      "behind the light front) are not on the device route")
        stage("setup")
        # ---- order >=2 source on the node bands (shower/api.py:373-402)
        frame = axis_frame(el["start_m"], el["direction"], el["length_m"], el["coefficient0"])
        pts_d, ch_d, npts_d, reference, frame = T.source.compile(el, frame)
        npts = npts_d.cpu().numpy()
        centre, axis, e1, e2 = (np.asarray(v, float) for v in frame)
        pts_host = pts_d.cpu().numpy()
        nb_bands = len(T.fold_bands)
        points = []
        for b in range(nb_bands):
            p = pts_host[b, :npts[b]]
            points.append(centre + p[:, :1] * axis + p[:, 1:2] * e1 + p[:, 2:3] * e2)
        if np.all(npts == npts[0]):
            channels = ch_d[:, :int(npts[0])]
        else:
            channels = [ch_d[b, :int(npts[b])] for b in range(nb_bands)]
        zero_ch = [ch_d[b, :int(npts[b]), :, 0].cpu().numpy() for b in range(nb_bands)]
        stage("source_compile")
        # ---- radial windows (shower/api.py:322-340, shower_basis.py:408-439)
        used = np.zeros(n, np.int64)
        near = np.zeros(n, bool)
        tail = np.zeros(n)
        weight_ratio = float(np.sum(T.fold_scale) / np.sum(T.fold_scale[T.fold_bands]))
        radius = None
        for b, band in enumerate(T.fold_bands):
            photons = np.sqrt(4 * np.pi) * np.abs(zero_ch[b][:, 0]) / T.efficiency[band]
            if radius is None or not np.array_equal(points[b], points[b - 1]):
                radius = np.sqrt(((points[b][None] - T.positions[:, None]) ** 2).sum(axis=2))
                n_near = np.count_nonzero(radius < low, axis=1)
                om, pt = np.nonzero(radius > high)
                n_far = np.bincount(om, minlength=n)
                far_factor = T.attenuation(radius[om, pt]) / (4 * np.pi * radius[om, pt] ** 2)
            used = np.maximum(used, len(points[b]) - n_near - n_far)
            near |= n_near > 0
            tail += weight_ratio * (10 * T.areas * T.peak_acceptance * T.efficiency[band]
                                    * np.bincount(om, weights=photons[pt] * far_factor,
                                                  minlength=n))
        if np.any(near):
            raise NotImplementedError("basis points inside the table's inner radius need the "
                                      "near-field clamp (near_field.py), not on the device route")
        reach = np.flatnonzero(used > 0)
        stage("radial_window")
        # ---- predictor (shower/ge2.py:70-96) and its zero-frequency charge
        predicted = np.zeros(n)
        late_charge = np.zeros(n)
        if len(reach):
            c_points, c_channels = [], []
            for b in range(nb_bands):
                rel = points[b] - centre
                coords = np.column_stack((rel @ axis, rel @ e1, rel @ e2))
                keys = np.floor(coords / float(cfg.predictor_cell_m)).astype(np.int64)
                _, inverse = np.unique(keys, axis=0, return_inverse=True)
                inverse = np.asarray(inverse).ravel()
                groups = int(inverse.max()) + 1
                wgt = np.abs(zero_ch[b][:, 0])
                total = np.bincount(inverse, weights=wgt, minlength=groups)
                count = np.bincount(inverse, minlength=groups)
                share = np.where(total[inverse] > 0, wgt / np.where(total > 0, total, 1.0)[inverse],
                                 1.0 / count[inverse])
                centroid = np.stack([np.bincount(inverse, weights=share * coords[:, k],
                                                 minlength=groups) for k in range(3)], axis=1)
                summed = np.zeros((groups, zero_ch[b].shape[1]), complex)
                np.add.at(summed, inverse, zero_ch[b])
                c_points.append(centre + centroid[:, :1] * axis + centroid[:, 1:2] * e1
                                + centroid[:, 2:3] * e2)
                c_channels.append(summed[:, :, None])
            if all(len(p) == len(c_points[0]) for p in c_points[1:]):
                c_ch = np.stack(c_channels)
            else:
                c_ch = c_channels
            predicted[reach] = self._apply(c_points, c_ch, reference, frame, reach,
                                           zero_frequency=True)[0].real
        stage("predictor")
        # ---- clocks (shower/api.py:455-477)
        fastest = float(np.min(T.group))
        time_width = float(np.ptp(edges))
        span = float(np.max(el["end_ns"]) - np.min(el["start_ns"]))
        mid = el["start_m"] + 0.5 * el["length_m"][:, None] * el["direction"]
        extent = float(np.linalg.norm(np.ptp(mid, axis=0)))
        local_origin = extent > high or span > 0.5 * time_width
        if time_origin_ns is not None:
            origins = np.asarray(time_origin_ns, float)
            if origins.shape != (n,) or not np.isfinite(origins).all():
                raise ValueError("time_origin_ns must hold one finite origin per OM")
        elif local_origin:
            origins = T.om_geometry(el, fastest, want_distance=False, want_earliest=True)[1]
        else:
            origins = (float(el["start_ns"][first])
                       + np.linalg.norm(T.positions - el["start_m"][first], axis=1)
                       / (C_M_PER_NS / fastest))
        safety = float(cfg.predictor_safety)
        prompt_extra = safety * np.abs(predicted) + np.abs(late_charge) + extra
        stage("clock")
        charge01, b1, computed, level1, prompt_el, bins0 = self._prompt(el, origins, prompt_extra,
                                                                        stage)
        # ---- exact zero-frequency >=2 where the decision needs it (shower/api.py:488-525)
        charge = np.zeros((n, 3))
        charge[:, :2] = charge01
        prompt_charge = charge[:, :2].sum(axis=1)
        computable = (used > 0) | (prompt_charge > 0)
        candidate = (used > 0) & (prompt_charge + safety * np.abs(predicted) + late_charge + extra
                                  >= threshold)
        if threshold == 0:
            candidate = used > 0
        zero_only = ([c[:, :, :1] for c in channels] if isinstance(channels, list)
                     else channels[:, :, :, :1])

        def exact(mask):
            ids = np.flatnonzero(mask)
            values = np.zeros(n)
            if len(ids):
                values[ids] = self._apply(points, zero_only, reference, frame, ids,
                                          zero_frequency=True)[0].real
            return values

        level = np.where(used > 0, 1, 0).astype(np.int8)
        exact_charge = exact(candidate)
        ratio = np.abs(exact_charge[candidate]) / np.maximum(np.abs(predicted[candidate]), 1e-300)
        fallback = bool(np.any(np.abs(exact_charge[candidate])
                               > safety * np.abs(predicted[candidate])))
        if fallback:
            candidate = used > 0
            exact_charge = exact(candidate)
        charge[:, 2] = predicted + late_charge
        charge[candidate, 2] = exact_charge[candidate] + late_charge[candidate]
        level[candidate] = 2
        active = computable & (charge.sum(axis=1) + extra >= threshold)
        if threshold == 0:
            active = computable
        if np.any(active & (level == 1)):
            raise RuntimeError("an OM was activated by a predicted >=2 charge")
        stage("ge2_exact_zero")
        # ---- full frequencies for the active OMs, then the readout
        spectrum = np.zeros((len(omega), n), complex)
        work = np.flatnonzero(active & (used > 0))
        if len(work):
            spectrum[:, work] = self._apply(points, channels, reference, frame, work,
                                            zero_frequency=False)
        stage("ge2_full")
        spectrum[0] = charge[:, 2] - late_charge
        components = np.zeros((n, len(edges) - 1, 3))
        if np.any(active):
            missing = np.flatnonzero(active & ~computed)
            if len(missing):
                # the reference recomputes the prompt without its screen (shower/api.py:592-599)
                q1m, b1m = self._fine_order1(prompt_el, origins, missing)
                charge[missing, 1] = q1m
                b1[missing] = b1m
            ids = np.flatnonzero(active)
            # order-0 bins of the active OMs (PreparedBallistic.bins, prompt.py:896-903);
            # their charge is the binned integral's, as in the reference
            components[ids, :, 0] = bins0[ids]
            components[ids, :, 1] = b1[ids]
            stage("order0_bins")
            rel = spectrum[:, ids] * np.exp(-1j * omega[:, None] * origins[None, ids])
            rel_t = torch.tensor(np.ascontiguousarray(rel.T).astype(np.complex64),
                                 device=T.device)
            bins2, _ = T.readout.bins(rel_t, mode=cfg.readout_mode)
            components[ids, :, 2] = bins2.cpu().numpy().astype(float)
        stage("readout")
        metadata = {
            "route": "lighthit_b200.shower", "ge2_charge_level": level.tolist(),
            "ge2_predictor": {"cell_m": float(cfg.predictor_cell_m), "safety": safety,
                              "candidates": int(candidate.sum()), "reachable": int(len(reach)),
                              "fallback_to_exact": fallback,
                              "exact_over_prediction_max": float(ratio.max(initial=0.0))},
            "prompt_order1_level": level1.tolist(), "radial_window_m": [low, high],
            "radial_tail_estimate_max_pe": float(tail.max(initial=0.0)),
            "time_origin": ("supplied event clock" if time_origin_ns is not None else
                            "earliest local segment and fastest group flight" if local_origin
                            else "earliest element start and fastest group flight"),
            "active_modules": int(active.sum()), "threshold_pe": threshold,
            "ge2_points": [int(v) for v in npts], "source_elements": len(el["beta"]),
            "elapsed_seconds": perf_counter() - began, "timings": stage.times}
        return HybridTransportResponse(None, omega.copy(), edges.copy(), spectrum, components,
                                       charge, origins, active, "shower", metadata)

    def _fine_order1(self, el, origins, ids):
        """Full-resolution order 1 (charge, bins) of the OMs ``ids``."""
        T = self.tables
        cone = float(np.sum(T.prompt["s0w"] * T.phase) / np.sum(T.prompt["s0w"]))
        table = pencils(T.order1, el, 1.0 / (el["beta"] * cone))
        q1, bins1 = grouped(T.order1, table, ids, origins)
        return q1.cpu().numpy()[ids], bins1.cpu().numpy()[ids]

    def _prompt(self, el, origins, extra, stage):
        """Orders 0 and 1 charges (``transport_prompt``, ``prompt.py:500-947``)."""
        T, cfg = self.tables, self.config
        n = T.n_om
        edges, threshold = T.edges, T.threshold
        valid = el["beta"] * T.threshold_phase > 1
        if not np.any(valid):
            raise ValueError("source is below Cherenkov threshold over the wavelength range")
        if not np.all(valid):
            el = _subset(el, valid)
        fastest = float(np.min(T.group))
        distance, _ = T.om_geometry(el, fastest)
        max_distance = T.radial[1]
        inside = distance <= max_distance
        s0 = 1.0 / T.wavelengths ** 2
        density = (el["coefficient0"][:, None] * s0[None]
                   + el["coefficient2"][:, None] * (s0 / T.phase ** 2)[None])
        emitted = float(np.sum(T.weights[None, :] * np.maximum(density, 0.0)))
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
        work = np.flatnonzero(inside)
        stage("prompt_selection")
        charge = np.zeros((n, 2))
        level = np.zeros(n, np.int8)
        if not len(work):
            empty = np.zeros((n, len(edges) - 1))
            return charge, empty, inside, level, el, empty
        # one order-0 pass gives the charge of every OM and the bins (PreparedBallistic.charge
        # and .bins integrate the same light; the route keeps the binned charge of active OMs)
        out0 = order0(T.order0, [el], origins[None], edges)
        q0 = out0["charge"][0].cpu().numpy()
        bins0 = out0["bins"][0]
        charge[work, 0] = q0[work]
        stage("order0_charge")
        # order 1: the fused unit of elements emitting in every band
        # (prompt.py:689-707, muon/secondary_first.py:184-204)
        if not np.all(el["beta"][:, None] * T.phase[None, :] > 1):
            raise NotImplementedError("elements above threshold in only some bands need the "
                                      "per-band order-1 units")
        cone = float(np.sum(T.prompt["s0w"] * T.phase) / np.sum(T.prompt["s0w"]))
        cone_cos = 1.0 / (el["beta"] * cone)
        # coarse charge screen and the reference's decision rule (prompt.py:720-812):
        # full resolution where q0 + extra + margin * q1_coarse reaches threshold
        fine_work = work
        coarse = None
        if cfg.screen and threshold > 0:
            coarse = grouped(T.order1_screen, pencils(T.order1_screen, el, cone_cos), work,
                             origins)[0].cpu().numpy()
            charge[work, 1] = coarse[work]
            level[work] = 1
            stage("order1_screen")
            fine_work = work[(charge[work, 0] + extra[work] + cfg.screen_margin
                              * np.maximum(coarse[work], 0.0)) >= threshold]
        b1 = np.zeros((n, len(edges) - 1))
        if len(fine_work):
            table = pencils(T.order1, el, cone_cos)
            q1, bins1 = grouped(T.order1, table, fine_work, origins)
            q1, bins1 = q1.cpu().numpy(), bins1.cpu().numpy()
            charge[fine_work, 1] = q1[fine_work]
            b1[fine_work] = bins1[fine_work]
            level[fine_work] = 2
            if coarse is not None:
                worst = float(np.min(coarse[fine_work] / np.maximum(q1[fine_work], 1e-300)))
                if worst * cfg.screen_margin < 1.0:
                    wider = 1.5 / max(worst, 1e-3)
                    more = work[(level[work] == 1) & (charge[work, 0] + extra[work] + wider
                                                      * np.maximum(coarse[work], 0.0)
                                                      >= threshold)]
                    if len(more):
                        q1, bins1 = grouped(T.order1, table, more, origins)
                        charge[more, 1] = q1.cpu().numpy()[more]
                        b1[more] = bins1.cpu().numpy()[more]
                        level[more] = 2
        stage("order1_fine")
        return charge, b1, level == 2, level, el, bins0.cpu().numpy()


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
    args = ap.parse_args(argv)
    route = ShowerTransport(ShowerTables.synthetic(args.tables), profile=args.profile)
    draws = shower_stream(args.showers, route.tables.positions.mean(axis=0))
    for d in draws:
        el = gaussian_shower(d["position_m"], d["direction"],
                             charged_track_length_m=d["charged_track_length_m"],
                             elements=d["elements"], seed=d["seed"])
        r = route(el)
        torch.cuda.synchronize()
        print(json.dumps({"elements": d["elements"], "active": int(r.active.sum()),
                          "charge_pe": float(r.charge_pe.sum()),
                          "ms": 1e3 * r.metadata["elapsed_seconds"]}), flush=True)


if __name__ == "__main__":
    main()
