"""Events of several sources on one clock with one OM selection (``EventTransport``).

Reference: ``EventTransport`` (``event.py:94-296``). Every source of an event
is transported on the event's clock (``common_time_origins``, the earliest
arrival from any step of any source at the fastest group speed), each with
the charge of the sources before it added to its threshold decisions; then,
in completion rounds, every OM whose summed charge (estimated scattered
charges inflated by ``safety``) can reach the threshold is recomputed in full
in every source that only estimated it (``receivers``). The response sums the
sources: charge and spectrum everywhere, bins where the sum is active.

The sources run through the device shower route (:class:`ShowerTransport`,
receiver subsets included) and calibration flashes through a flash transport;
this module is the host orchestration of those calls, as in the reference.
Muon components need the reference's muon route and its tables, which are not
on the device: they raise ``NotImplementedError``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from time import perf_counter

import numpy as np

from .shower import HybridTransportResponse, elements_of

__all__ = ["SourceComponent", "EventTransport", "common_time_origins"]


@dataclass
class SourceComponent:
    """One light source of an event (``event.py:40-62``)."""
    kind: str
    source: object
    ancestry: dict | None = None
    primary_uid: int | None = None
    label: str = ""

    def __post_init__(self):
        if self.kind not in ("shower", "muon"):
            raise ValueError("component kind must be 'shower' or 'muon'")
        if self.kind == "muon" and (self.ancestry is None or self.primary_uid is None):
            raise ValueError("a muon component needs ancestry and primary_uid")


@dataclass
class _Part:
    component: SourceComponent
    charge: np.ndarray
    bins: np.ndarray
    spectrum: np.ndarray
    detailed: np.ndarray
    runs: list = field(default_factory=list)


def common_time_origins(tables, sources):
    """``common_time_origins`` (``event.py:65-80``): per OM, the earliest arrival
    from any step of ``sources`` at the fastest group speed (device, float64)."""
    group = float(np.min(tables.group))
    origins = np.full(tables.n_om, np.inf)
    for source in sources:
        _, early = tables.om_geometry(elements_of(source), group, want_distance=False,
                                      want_earliest=True)
        origins = np.minimum(origins, early)
    return origins


class EventTransport:
    """``EventTransport(kernel, *, muon_data=None, shower_data=None, laser_kernel=None,
    threads=None, safety=3.0, max_rounds=4)(components | IsotropicFlash)`` on the
    device routes (``event.py:94-296``).

    ``kernel``: the device shower route (a :class:`lighthit_b200.shower.ShowerTransport`),
    its tables (:class:`~lighthit_b200.shower.ShowerTables`), or the reference's
    ``TransportKernel`` (the shower route is then built from ``shower_data`` as
    the reference's ``shower_route`` does, ``event.py:124-129``).
    ``laser_kernel``: a flash transport (:class:`lighthit_b200.flash.FlashTransport`
    or :class:`~lighthit_b200.flash.BroadbandFlashTransport`) for calibration
    flashes; ``flash`` is the same argument under its earlier name.
    ``muon_data`` and ``threads`` are accepted for the reference's signature:
    muon components raise ``NotImplementedError`` (the muon route is not on the
    device) and the device routes take no thread count.
    """

    def __init__(self, kernel, *, muon_data=None, shower_data=None, laser_kernel=None,
                 threads=None, safety=3.0, max_rounds=4, flash=None):
        from .shower import ShowerTables, ShowerTransport
        if not np.isfinite(safety) or safety < 1 or int(max_rounds) < 1:
            raise ValueError("safety must be >= 1 and max_rounds positive")
        if isinstance(kernel, ShowerTransport):
            self.shower = kernel
        elif isinstance(kernel, ShowerTables):
            self.shower = ShowerTransport(kernel)
        else:
            self.shower = ShowerTransport(kernel, shower_data, threads=threads)
        self.kernel = kernel
        self.muon_data, self.shower_data, self.threads = muon_data, shower_data, threads
        self.flash_transport = laser_kernel if laser_kernel is not None else flash
        self.safety, self.max_rounds = float(safety), int(max_rounds)
        self.route_fallbacks = {}

    def shower_route(self):
        """The device shower route (``event.py:124-129``)."""
        return self.shower

    def _run(self, component, **options):
        if component.kind != "shower":
            raise NotImplementedError("muon components need the reference's muon route "
                                      "(MuonTransport) and its tables")
        return self.shower(component.source, **options)

    def flash(self, flash):
        """A calibration flash, transported alone (``event.py:184-190``)."""
        if self.flash_transport is None:
            raise ValueError("a calibration flash needs EventTransport(laser_kernel=...)")
        response = self.flash_transport.transport(flash)
        response.metadata["route"] = "lighthit_b200.flash (isotropic flash)"
        return response

    def __call__(self, components):
        from .model import IsotropicFlash
        if isinstance(components, IsotropicFlash) or hasattr(components, "spectral_shape"):
            return self.flash(components)
        components = list(components)
        if not components:
            raise ValueError("an event needs at least one source component")
        if any(isinstance(c, IsotropicFlash) or hasattr(c, "spectral_shape") for c in components):
            raise ValueError("a calibration flash is transported alone (different kernel)")
        if len(components) == 1:
            response = self._run(components[0])
            response.metadata["event_components"] = [self._describe(components[0])]
            return response
        return self._compose(components)

    @staticmethod
    def _describe(component):
        return dict(kind=component.kind, label=component.label,
                    elements=len(elements_of(component.source)["beta"]),
                    primary_uid=component.primary_uid)

    def _compose(self, components):
        """Several sources on one clock with one OM selection (``event.py:193-296``)."""
        began = perf_counter()
        tables = self.shower.tables
        n = tables.n_om
        edges = np.asarray(tables.edges, float)
        threshold = float(tables.threshold)
        origins = common_time_origins(tables, [c.source for c in components])
        order = sorted(range(len(components)), key=lambda i: components[i].kind != "shower")
        parts = [None] * len(components)
        known = np.zeros(n)
        omega = None
        for index in order:
            component = components[index]
            response = self._run(component, time_origin_ns=origins, selection_extra_charge=known)
            if omega is None:
                omega = np.asarray(response.omega_per_ns)
            if not np.allclose(response.time_origin_ns, origins, rtol=0, atol=1e-9):
                raise ValueError(f"{component.kind} route did not use the event clock")
            charge = np.asarray(response.charge_components_pe, float).copy()
            detailed = np.asarray(response.active, bool).copy()
            # a source that does not reach an OM contributes exactly nothing there
            detailed |= np.all(charge == 0.0, axis=1)
            part = _Part(component, charge,
                         np.where(detailed[:, None, None], response.components_pe, 0.0),
                         np.asarray(response.spectrum_ge2_pe).copy(), detailed)
            part.runs.append(dict(receivers="all",
                                  route_active=int(np.count_nonzero(response.active))))
            parts[index] = part
            known += part.charge.sum(axis=1)
        rounds = []
        for round_number in range(self.max_rounds):
            upper = np.zeros(n)
            for part in parts:
                q = part.charge
                inflated = np.maximum(q[:, 0], 0.0) + self.safety * np.abs(q[:, 1:]).sum(axis=1)
                upper += np.where(part.detailed, q.sum(axis=1), inflated)
            wanted = upper >= threshold
            done = True
            record = dict(round=round_number, candidates=int(wanted.sum()), recomputed={})
            for part in parts:
                need = np.flatnonzero(wanted & ~part.detailed
                                      & (np.abs(part.charge).sum(axis=1) > 0))
                if not len(need):
                    continue
                done = False
                local = self._run(part.component, time_origin_ns=origins[need],
                                  selection_extra_charge=None, receivers=need)
                part.charge[need] = local.charge_components_pe
                part.bins[need] = local.components_pe
                part.spectrum[:, need] = local.spectrum_ge2_pe
                part.detailed[need] = True
                part.runs.append(dict(receivers=need.tolist()))
                record["recomputed"][part.component.label or part.component.kind] = len(need)
            rounds.append(record)
            if done:
                break
        else:
            raise RuntimeError("source composition did not converge; raise max_rounds")
        charge = sum(part.charge for part in parts)
        detailed = np.logical_and.reduce([part.detailed for part in parts])
        active = (charge.sum(axis=1) >= threshold) & detailed
        if threshold == 0:
            active = detailed & (np.abs(charge).sum(axis=1) > 0)
        if np.any((charge.sum(axis=1) >= threshold) & ~detailed):
            raise RuntimeError("an OM above threshold lacks the detailed charge of a source")
        components_pe = np.zeros((n, len(edges) - 1, 3))
        components_pe[active] = sum(part.bins for part in parts)[active]
        spectrum = sum(part.spectrum for part in parts)
        metadata = dict(
            route="lighthit_b200.event", elapsed_seconds=perf_counter() - began,
            threshold_pe=threshold,
            time_origin="earliest arrival from any step of the event, fastest group speed",
            selection="summed charge of all sources; OMs completed in every source while "
                      "q0 + safety*(|q1|+|q2|) of estimated sources can reach the threshold",
            safety=self.safety, completion_rounds=rounds, active_modules=int(active.sum()),
            event_components=[dict(self._describe(part.component), runs=part.runs,
                                   charge_pe=float(part.charge.sum()),
                                   detailed_modules=int(part.detailed.sum()))
                              for part in parts],
            inactive_charge_may_be_estimated=bool(np.any(~detailed)),
            computed_orders=[0, 1, ">=2"])
        return HybridTransportResponse(None, omega, edges, spectrum, components_pe, charge,
                                       origins, active, "event", metadata)
