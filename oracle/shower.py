"""Oracle: the whole shower route on the CPU. Test infrastructure only.

Restates ``transport_shower`` (``shower/api.py:221-539``) with
``transport_prompt`` (``prompt.py:500-947``) in float64 on the host:

* source preparation and the order >=2 contraction: ``oracle.source``
  (``node_sources``, ``collapse``) and ``oracle.ge2.apply_folded`` (C loops);
* radial windows and the far-tail estimate (``shower_basis.py:388-439``);
* clocks (``shower/api.py:355-376``, ``earliest_element_arrival``,
  ``_shower_basis.py:50-78``);
* module selection (``prompt.py:603-631``), order 0 by the first-entry ray
  quadrature with the Gauss order doubled until it converges
  (``oracle.order0.direct_light``), order 1 by the fused-band grouped pencils
  with the global coarse screen and its widening (``prompt.py:670-812``,
  ``oracle.order1``);
* the predictor, the exact zero-frequency charge and its fallback, ``active``,
  the full spectrum of the active OMs and its readout (``shower/api.py:339-421``,
  ``oracle.readout``);
* delayed light (``shower/ge2.py:122-147``, ``shower/api.py:294-310, 402-421``).

Tables are the route's reference-built constants (``route_<config>.npz``), its
folded >=2 kernels and, for showers passing closer than the radial minimum,
the near-field interval (``oracle.near``).
"""
from __future__ import annotations

import numpy as np

from . import order0 as O0
from . import order1 as O1
from . import source as S
from .ge2 import apply_folded as _apply
from .readout import readout_bins

C_M_PER_NS = 0.299792458
ELEMENT_KEYS = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
                "start_ns", "end_ns")


def _subset(el, mask):
    return {k: v[mask] for k, v in el.items()}


def delay_groups(el, *, prompt_delay_ns, cell_ns, window_end_ns, group_index_max):
    """``delay_groups`` (``shower/ge2.py:122-147``)."""
    first = int(np.argmin(el["start_ns"]))
    distance = np.linalg.norm(el["start_m"] - el["start_m"][first], axis=1)
    delay = el["start_ns"] - el["start_ns"][first] - distance / C_M_PER_NS
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


def earliest_element_arrival(receivers, el, group_index):
    """``earliest_element_arrival`` (``_shower_basis.py:50-78``)."""
    flight = float(group_index) / C_M_PER_NS
    out = np.empty(len(receivers))
    for r, pos in enumerate(receivers):
        d = pos[None, :] - el["start_m"]
        along = np.clip((d * el["direction"]).sum(axis=1), 0.0, el["length_m"])
        d = d - along[:, None] * el["direction"]
        out[r] = np.min(el["start_ns"] + flight * np.sqrt((d * d).sum(axis=1)))
    return out


def min_distance_to_segments(receivers, el):
    """``min_distance_to_segments`` (``_prompt_numba.py``): closest approach of
    every OM to any element segment."""
    out = np.empty(len(receivers))
    for r, pos in enumerate(receivers):
        d = pos[None, :] - el["start_m"]
        along = np.clip((d * el["direction"]).sum(axis=1), 0.0, el["length_m"])
        d = d - along[:, None] * el["direction"]
        out[r] = np.sqrt((d * d).sum(axis=1)).min()
    return out


class Route:
    """The route's reference-built tables (route constants, folded kernels, near field)."""

    def __init__(self, route, folded, near=None, *, order0_gauss=None, threads=1):
        """``order0_gauss``: None doubles the first-entry Gauss order from 8
        until every OM converges (the reference's tolerance, raising at 64 as
        ``_surface_ballistic.py:195-196`` does); an integer evaluates that order
        once (order 8 agrees with the reference's control-variate order 0 to
        about 3e-8 in charge on the README shower)."""
        self.order0_gauss = order0_gauss
        # OM-parallel stages run their C loops on `threads` threads over
        # interleaved OM subsets (the reference's prange over receivers); the
        # C calls release the interpreter lock
        self.threads = max(1, int(threads))
        self._pool = None
        self.r = {k: np.asarray(v) for k, v in dict(route).items()}
        self.folded = {k: np.asarray(v) for k, v in dict(folded).items()}
        self.near = None if near is None else {k: np.asarray(v) for k, v in dict(near).items()}
        r = self.r
        self.positions = r["positions_m"].astype(float)
        self.looks = r["looks"].astype(float)
        self.areas = r["areas_m2"].astype(float)
        self.alpha = r["alpha"].astype(float)
        self.omega = r["omega_per_ns"].astype(float)
        self.edges = r["edges_ns"].astype(float)
        self.threshold = float(r["threshold_pe"])
        self.low, self.high = (float(v) for v in r["radial_range_m"])
        w = r["weight_nm"] * r["efficiency"] / r["wavelength_nm"] ** 2
        lowest = float(r["absorption_per_m"].min())
        radius = np.geomspace(1e-3, 1e5, 1025)
        log_factor = (np.log(np.exp(-np.outer(radius, r["absorption_per_m"] - lowest)) @ w / w.sum())
                      - lowest * radius)
        self.attenuation = lambda d: np.exp(np.interp(d, radius, log_factor))
        self.zero = dict(self.folded, coefficients=self.folded["coefficients"][..., :1],
                         omega=self.folded["omega"][:1])
        self.monomials = O1.acceptance_monomials(self.alpha)

    def _map(self, fn, ids):
        """``fn(chunk)`` over interleaved chunks of ``ids``: [(chunk, result)]."""
        ids = np.asarray(ids)
        if self.threads == 1 or len(ids) < 2:
            return [(ids, fn(ids))]
        chunks = [ids[k::self.threads] for k in range(self.threads) if len(ids[k::self.threads])]
        if self._pool is None:
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(self.threads)
        return list(zip(chunks, self._pool.map(fn, chunks)))

    # ---- order >=2 helpers
    def _sources(self, el, omega, frame):
        r = self.r
        return S.node_sources(el, r["wavelength_nm"], r["fold_phase"], r["fold_scale"],
                              r["fold_bands"], int(r["source_degree"]), int(r["azimuthal_degree"]),
                              omega, frame)

    def apply(self, folded, sources, ids):
        """``apply_folded`` (``shower/ge2.py:99-119``) at the OMs ``ids``: (W, len(ids))."""
        ids = np.asarray(ids)
        if not len(ids):
            return np.zeros((len(folded["omega"]), 0), complex)
        out = np.zeros((len(folded["omega"]), len(ids)), complex)
        where = {int(v): k for k, v in enumerate(ids)}
        for chunk, res in self._map(lambda c: self._apply_ids(folded, sources, c), ids):
            out[:, [where[int(v)] for v in chunk]] = res
        return out

    def _apply_ids(self, folded, sources, ids):
        pos, looks, area = self.positions[ids], self.looks[ids], self.areas[ids]
        centre, axis, first, second = sources[0].frame
        frame = dict(centre=centre, first=first, second=second, axis=axis)
        pts = sources[0].points_m()
        window = (self.low, self.high)
        if all(np.array_equal(s.points_m(), pts) for s in sources[1:]):
            src = dict(points_m=pts, channels=np.stack([s.channels for s in sources]),
                       reference_ns=np.array([s.reference_ns for s in sources]), frame=frame,
                       degree=int(self.r["source_degree"]),
                       azimuthal_degree=int(self.r["azimuthal_degree"]))
            return _apply(folded, src, pos, looks, self.alpha, area, window, fast=True)
        total = 0
        for j, s in enumerate(sources):
            band = dict(folded, coefficients=folded["coefficients"][j:j + 1],
                        absorption=folded["absorption"][j:j + 1], speed=folded["speed"][j:j + 1])
            src = dict(points_m=s.points_m(), channels=s.channels[None],
                       reference_ns=np.array([s.reference_ns]), frame=frame,
                       degree=int(self.r["source_degree"]),
                       azimuthal_degree=int(self.r["azimuthal_degree"]))
            total = total + _apply(band, src, pos, looks, self.alpha, area, window, fast=True)
        return total

    # ---- orders 0 and 1 (transport_prompt)
    def prompt(self, el, extra, origins, local_origin):
        r = self.r
        n = len(self.positions)
        thr = self.threshold
        valid = el["beta"] * float(r["threshold_phase"]) > 1
        if not np.any(valid):
            raise ValueError("source is below Cherenkov threshold over the wavelength range")
        pel = el if np.all(valid) else _subset(el, valid)
        fastest = float(np.min(r["group_index"]))
        if not local_origin:
            first = int(np.argmin(pel["start_ns"]))
            origins_p = (float(pel["start_ns"][first])
                         + np.linalg.norm(self.positions - pel["start_m"][first], axis=1)
                         / (C_M_PER_NS / fastest))
            if not np.allclose(origins_p, origins, rtol=0, atol=1e-10):
                raise ValueError("prompt and RTE time origins differ")
        distance = min_distance_to_segments(self.positions, pel)
        inside = distance <= self.high
        lam, ph = r["wavelength_nm"], r["phase_index"]
        density = (pel["coefficient0"][:, None] / lam[None, :] ** 2
                   + pel["coefficient2"][:, None] / (lam[None, :] ** 2 * ph[None, :] ** 2))
        emitted = float(np.sum(r["weight_nm"][None, :] * np.maximum(density, 0.0)))
        far = np.maximum(distance, 1e-9)
        upper = (10 * max(emitted, 0.0) * self.areas * float(r["peak_acceptance"])
                 * float(np.max(r["efficiency"])) * np.exp(-float(np.min(r["absorption_per_m"])) * far)
                 / (4 * np.pi * far ** 2))
        unsafe = (~inside) & (upper >= thr)
        if np.any(unsafe):
            raise ValueError(f"{int(unsafe.sum())} OMs beyond max_distance_m={self.high:g} have a "
                             "conservative estimate above threshold; increase max_distance_m")
        too_close = inside & (distance < 0.1)
        if np.any(too_close):
            raise ValueError(f"{int(too_close.sum())} OMs are closer than min_distance_m=0.1 m "
                             "to the source")
        work = np.flatnonzero(inside)
        charge = np.zeros((n, 2))
        bins = np.zeros((n, len(self.edges) - 1, 2))
        # order 0: first-entry rays, Gauss order doubled until it converges
        if len(work):
            det = dict(positions_m=self.positions[work], looks=self.looks[work],
                       areas_m2=self.areas[work], radii_m=r["radii_m"][work], alpha=self.alpha)
            optics = {k: r[f"optics_{k}"] for k in ("panel_edges", "phase_nodes", "group_nodes",
                                                     "extinction_nodes", "efficiency_coefficients")}
            def order0(rows):
                sub = {k: v[rows] for k, v in det.items() if k != "alpha"}
                sub["alpha"] = self.alpha
                po, pe = O0.candidates(sub["positions_m"], sub["radii_m"], pel["start_m"],
                                       pel["direction"], pel["length_m"], pel["coefficient0"],
                                       pel["beta"], optics["phase_nodes"])
                if self.order0_gauss is None:
                    return O0.direct_light(po, pe, sub, pel, optics, origins[work][rows],
                                           self.edges)[:2]
                return O0.rays(po, pe, sub, pel, optics, origins[work][rows], self.edges,
                               int(self.order0_gauss))

            for rows, (q0, b0) in self._map(order0, np.arange(len(work))):
                charge[work[rows], 0] = q0
                bins[work[rows], :, 0] = b0
        # order 1: fused-band units with the global coarse screen
        bands = {k: r[k] for k in ("mus", "mut", "speed", "s0w", "s2w")}
        cone = float(np.sum(r["s0w"] * ph) / np.sum(r["s0w"]))
        everywhere = pel["beta"] * float(np.min(ph)) > 1
        units = []
        if np.any(everywhere):
            sub = pel if np.all(everywhere) else _subset(pel, everywhere)
            units.append((sub, 1.0 / (sub["beta"] * cone), bands, 96, 192))
        for b, phase in enumerate(ph):
            mask = (pel["beta"] * float(phase) > 1) & ~everywhere
            if np.any(mask):
                sub = _subset(pel, mask)
                units.append((sub, 1.0 / (sub["beta"] * float(phase)),
                              {k: v[b:b + 1] for k, v in bands.items()}, 32, 96))
        q1 = np.zeros(n)
        b1 = np.zeros((n, len(self.edges) - 1))
        level = np.zeros(n, np.int8)
        args = (self.positions, self.looks, self.areas, origins)
        screen = thr > 0
        fine_work = work
        coarse_total = None
        if screen and len(work):
            for sub, cone_cos, tab, _, _ in units:
                pack = O1.screen_pencils(sub, cone_cos)
                for ids, (q, _, _, _) in self._map(
                        lambda c, pack=pack, tab=tab: O1.grouped(
                            pack, *args, c, self.monomials, float(r["g"]), tab, self.edges,
                            merge=(2e-3, 0.3, 2.0, 0.02), compute_bins=False), work):
                    q1[ids] += q[ids]
            level[work] = 1
            coarse_total = q1.copy()
            fine_work = work[(charge[work, 0] + extra[work]
                              + 3.0 * np.maximum(q1[work], 0.0)) >= thr]
            q1[fine_work] = 0.0
        tables = []
        for sub, cone_cos, tab, face, ring in units:
            tables.append(O1.compress(sub, cone_cos, pixel_face=face, ring_nodes=ring))

        def fine(ids):
            q = np.zeros(n)
            b = np.zeros((n, len(self.edges) - 1))
            for (sub, cone_cos, tab, _, _), pen in zip(units, tables):
                for part, (qq, bb, _, _) in self._map(
                        lambda c, pen=pen, tab=tab: O1.grouped(
                            pen, *args, c, self.monomials, float(r["g"]), tab, self.edges), ids):
                    q[part] += qq[part]
                    b[part] += bb[part]
            return q, b

        if len(fine_work):
            q, b = fine(fine_work)
            q1[fine_work] += q[fine_work]
            b1 += b
            level[fine_work] = 2
        if screen and len(fine_work):
            ratio = coarse_total[fine_work] / np.maximum(q1[fine_work], 1e-300)
            worst = float(np.min(ratio))
            if worst * 3.0 < 1.0:
                wider = 1.5 / max(worst, 1e-3)
                more = work[(level[work] == 1) & (charge[work, 0] + extra[work]
                                                   + wider * np.maximum(coarse_total[work], 0.0)
                                                   >= thr)]
                if len(more):
                    q, b = fine(more)
                    q1[more] = q[more]
                    b1[more] += b[more]
                    level[more] = 2
        charge[:, 1] = q1
        active = inside & (charge.sum(axis=1) + extra >= thr)
        if thr == 0:
            active = inside.copy()
        if np.any(active & (level < 2)):
            raise ValueError("prompt screen omitted an OM selected by the combined charge")
        bins[:, :, 1] = b1
        bins[~active] = 0.0
        return dict(charge=charge, bins=bins, active=active, computed=inside, level=level,
                    elements=pel)

    # ---- the route
    def __call__(self, elements, *, time_origin_ns=None, selection_extra_charge=None):
        r = self.r
        el = {k: np.asarray(elements[k], float) for k in ELEMENT_KEYS}
        n = len(self.positions)
        omega, edges, thr = self.omega, self.edges, self.threshold
        phase, group = r["phase_index"], r["group_index"]
        max_phase = float(np.max(phase))
        valid = el["beta"] * max_phase > 1
        if not np.any(valid):
            raise ValueError("source is below Cherenkov threshold over the wavelength range")
        if not np.all(valid):
            el = _subset(el, valid)
        extra = (np.zeros(n) if selection_extra_charge is None
                 else np.maximum(np.asarray(selection_extra_charge, float), 0.0))
        prompt_mask, late_groups, beyond = delay_groups(
            el, prompt_delay_ns=20.0, cell_ns=20.0, window_end_ns=float(edges[-1]),
            group_index_max=float(np.max(group)))

        def compiled(mask, frequencies):
            part = el if np.all(mask) else _subset(el, mask)
            return self._sources(part, frequencies, S.axis_frame(part, part["coefficient0"]))

        sources = compiled(prompt_mask, omega)
        late_zero = compiled(~prompt_mask, omega[:1]) if np.any(~prompt_mask) else None
        late_sources = [(shift, compiled(mask, omega)) for mask, shift in late_groups]
        # radial windows
        used = np.zeros(n, np.int64)
        near = np.zeros(n, bool)
        tail = np.zeros(n)
        fold_bands, fold_scale = r["fold_bands"], r["fold_scale"]
        weight_ratio = float(np.sum(fold_scale) / np.sum(fold_scale[list(fold_bands)]))
        for group_sources in [sources] + ([late_zero] if late_zero is not None else []):
            for band, item in zip(fold_bands, group_sources):
                eff = float(r["efficiency"][band])
                photons = np.sqrt(4 * np.pi) * np.abs(item.channels[:, 0, 0]) / eff
                radius = np.linalg.norm(item.points_m()[None] - self.positions[:, None], axis=2)
                n_near = np.count_nonzero(radius < self.low, axis=1)
                far_mask = radius > self.high
                part_used = len(photons) - n_near - np.count_nonzero(far_mask, axis=1)
                distance = np.where(far_mask, radius, 1.0)
                tail += weight_ratio * (10 * self.areas * float(r["peak_acceptance"]) * eff * np.sum(
                    np.where(far_mask, photons[None] * self.attenuation(distance)
                             / (4 * np.pi * distance ** 2), 0.0), axis=1))
                near |= n_near > 0
                used = np.maximum(used, part_used)
        reach = np.flatnonzero(used > 0)
        predicted = np.zeros(n)
        late_charge = np.zeros(n)
        collapsed = S.collapse(sources, 2.0)
        if len(reach):
            predicted[reach] = self.apply(self.zero, collapsed, reach)[0].real
            if late_zero is not None:
                late_charge[reach] = self.apply(self.zero, late_zero, reach)[0].real
        # clocks
        fastest = float(np.min(group))
        time_width = float(np.ptp(edges))
        span = float(np.max(el["end_ns"]) - np.min(el["start_ns"]))
        mid = el["start_m"] + 0.5 * el["length_m"][:, None] * el["direction"]
        extent = float(np.linalg.norm(np.ptp(mid, axis=0)))
        local_origin = extent > self.high or span > 0.5 * time_width
        if time_origin_ns is not None:
            origins = np.asarray(time_origin_ns, float)
            local_origin = True
        elif local_origin:
            origins = earliest_element_arrival(self.positions, el, fastest)
        else:
            first = int(np.argmin(el["start_ns"]))
            origins = (float(el["start_ns"][first])
                       + np.linalg.norm(self.positions - el["start_m"][first], axis=1)
                       / (C_M_PER_NS / fastest))
        safety = 2.0
        prompt = self.prompt(el, safety * np.abs(predicted) + np.abs(late_charge) + extra, origins,
                             local_origin)
        charge = np.zeros((n, 3))
        charge[:, :2] = prompt["charge"]
        prompt_charge = charge[:, :2].sum(axis=1)
        computable = (used > 0) | (prompt_charge > 0)
        candidate = (used > 0) & (prompt_charge + safety * np.abs(predicted) + late_charge + extra
                                  >= thr)
        if thr == 0:
            candidate = used > 0
        zero_sources = [S.AxialSource(s.frame, s.z_m, s.transverse_m,
                                      np.ascontiguousarray(s.channels[:, :, :1]), s.reference_ns)
                        for s in sources]

        def exact(mask):
            ids = np.flatnonzero(mask)
            values = np.zeros(n)
            if len(ids):
                values[ids] = self.apply(self.zero, zero_sources, ids)[0].real
            return values

        level = np.where(used > 0, 1, 0).astype(np.int8)
        exact_charge = exact(candidate)
        fallback = bool(np.any(np.abs(exact_charge[candidate])
                               > safety * np.abs(predicted[candidate])))
        if fallback:
            candidate = used > 0
            exact_charge = exact(candidate)
        charge[:, 2] = predicted + late_charge
        charge[candidate, 2] = exact_charge[candidate] + late_charge[candidate]
        level[candidate] = 2
        active = computable & (charge.sum(axis=1) + extra >= thr)
        if thr == 0:
            active = computable
        if np.any(active & (level == 1)):
            raise RuntimeError("an OM was activated by a predicted >=2 charge")
        spectrum = np.zeros((len(omega), n), complex)
        work = np.flatnonzero(active & (used > 0))
        if len(work):
            spectrum[:, work] = self.apply(self.folded, sources, work)
        late_spectra = []
        for shift, group_sources in late_sources:
            values = np.zeros((len(omega), n), complex)
            if len(work):
                values[:, work] = self.apply(self.folded, group_sources, work)
            late_spectra.append((shift, values))
        spectrum[0] = charge[:, 2] - late_charge
        components = np.zeros((n, len(edges) - 1, 3))
        if np.any(active):
            if not np.all(prompt["active"][active]):
                raise ValueError("prompt bins are missing for an active OM")
            components[active, :, :2] = prompt["bins"][active]
            readout = r["readout_omega_per_ns"]
            relative = spectrum[:, active] * np.exp(-1j * omega[:, None] * origins[None, active])
            components[active, :, 2] = readout_bins(omega, relative, edges, readout)
            for shift, values in late_spectra:
                relative = values[:, active] * np.exp(-1j * omega[:, None]
                                                      * (origins[None, active] + shift))
                components[active, :, 2] += readout_bins(omega, relative, edges - shift, readout)
        out = dict(charge_components_pe=charge, components_pe=components, spectrum_ge2_pe=spectrum,
                   time_origin_ns=origins, active=active, ge2_charge_level=level,
                   prompt_order1_level=prompt["level"], fallback=fallback, near=near)
        if np.any(near):
            if self.near is None:
                raise NotImplementedError("the shower passes inside the radial minimum: the "
                                          "near-field table is needed")
            from .near import near_field
            oms, q_near, s_near, _ = near_field(
                self.near, el, self.positions, self.looks, self.areas, origins,
                wavelength_nm=r["wavelength_nm"], weight_nm=r["weight_nm"],
                efficiency=r["efficiency"], phase_index=r["phase_index"], alpha=self.alpha)
            # add_near_field (near_field.py:174-217): charge of every near OM,
            # bins of the active ones, the stored spectrum on the absolute clock
            charge[oms, 2] += q_near[oms]
            detailed = oms[active[oms]]
            if len(detailed):
                components[detailed, :, 2] += readout_bins(omega, s_near[:, detailed], edges,
                                                           r["readout_omega_per_ns"])
            spectrum[:, oms] += s_near[:, oms] * np.exp(1j * omega[:, None] * origins[None, oms])
            out["near_field_oms"] = oms
        return out
