"""The near-field clamp of order >=2 on the B200 (``near_field.py:91-217``).

The order >=2 tables start at a radial minimum (2 m here). Source points
closer than that to an OM are left out of the route's order >=2 sums and added
back here with the reference's clamp: the Green function at the radial minimum
along the same directions, with the flight phase of the actual distance
(``_cone_many_looks`` with ``clamp_low = 0``,
``muon/track_ge2_primitive.py:612-660``). The portions of the elements within
the radius of each OM (``near_portions``, ``near_field.py:39-69``), their
Gauss panels, the geometry and the contraction with the first radial interval
of the per-wavelength splines run in ``lh_near_field``; the table
(``tables/near_<config>.npz``) is that interval of ``Ge2KernelStore.bundle``,
written once by ``tables/build_tables.py``.

``add_near_field`` adds the result to a response as the reference does
(``near_field.py:174-217``): order >=2 charge of every near OM, bins where the
OM is active, the stored spectrum, ``metadata['near_field']`` and a
``RuntimeWarning`` naming the OMs.
"""
from __future__ import annotations

import ctypes as C
import warnings

import numpy as np

from . import _lib
from .ge2 import _start_norm

__all__ = ["NearTable", "NearField", "add_near_field"]

APPROXIMATION = ("order >=2 Green function clamped at the table radial minimum along the same "
                 "directions; flight time of the actual distance")


class NearField:
    """``NearFieldGe2`` (``near_field.py:30-36``): the clamped order >=2 of the near
    portions. ``spectrum`` is the device (OM, frequency) complex128 spectrum
    relative to the response clock (zero for OMs without portions)."""

    def __init__(self, oms, charge_pe, spectrum, metadata):
        self.oms = oms
        self.charge_pe = charge_pe
        self.spectrum = spectrum
        self.metadata = metadata


class NearTable:
    """The near-field inputs resident on the device: the first radial interval of
    every wavelength's order >=2 spline and the spectral constants."""

    def __init__(self, near, *, wavelength_nm, weight_nm, efficiency, phase_index, alpha,
                 panel_m=0.05, gauss_order=6, device="cuda"):
        import torch
        self.device = torch.device(device)
        dev = self.device
        z = dict(np.load(near)) if not isinstance(near, dict) else near
        coef = np.ascontiguousarray(z["coefficients"], np.complex64)
        self.n_lambda, deg1, self.n_pairs, _, self.n_omega = coef.shape
        self.degree = int(z["degree"])
        self.acc_degree = int(z["acceptance_degree"])
        if deg1 != self.degree + 1:
            raise ValueError("near-field table degree mismatch")
        self.log_r = np.asarray(z["log_r"], float)
        self.radial_minimum = float(np.exp(self.log_r[0]))
        self.omega = np.asarray(z["omega"], float)
        self.panel_m, self.gauss_order = float(panel_m), int(gauss_order)
        wl = np.asarray(wavelength_nm, float)
        if len(wl) != self.n_lambda:
            raise ValueError("near-field table and route wavelengths differ")
        nodes, weights = np.polynomial.legendre.leggauss(self.gauss_order)

        def f64(x):
            return torch.tensor(np.ascontiguousarray(x, float), dtype=torch.float64, device=dev)

        def i32(x):
            return torch.tensor(np.ascontiguousarray(x, np.int32), dtype=torch.int32, device=dev)

        self._coef = torch.view_as_real(torch.from_numpy(coef)).contiguous().to(dev)
        self._keep = [
            f64(z["absorption"]), f64(z["speed"]), f64(self.omega), i32(z["pair_lambda"]),
            i32(z["pair_mu"]), f64(np.asarray(alpha, float)[:self.acc_degree + 1]),
            f64(_start_norm(self.acc_degree)), f64(wl), f64(phase_index),
            f64(np.asarray(weight_nm, float) * np.asarray(efficiency, float)), f64(nodes),
            f64(weights)]
        k = [t.data_ptr() for t in self._keep]
        self.struct = _lib.NearTable(
            self.n_lambda, self.degree, self.acc_degree, self.n_pairs, self.n_omega,
            self._coef.data_ptr(), float(self.log_r[0]), float(self.log_r[1]),
            float(z["radial_high_m"]), k[0], k[1], k[2], k[3], k[4], k[5], k[6],
            int(str(z.get("phase", "flight")) == "flight"), k[7], k[8], k[9], self.gauss_order,
            k[10], k[11], self.panel_m)
        self._workspace = None

    def field(self, elements, n_elements, positions, looks, areas, origins, *, radius_m=None):
        """``near_field_ge2`` (``near_field.py:91-171``) for device element arrays
        ``elements`` (the reference's field names, float64) and device OM arrays;
        ``origins`` the response's per-OM clock (device float64)."""
        import torch
        dev = self.device
        n_om = int(positions.shape[0])
        radius = self.radial_minimum if radius_m is None else float(radius_m)
        spectrum = torch.empty((n_om, self.n_omega), dtype=torch.complex128, device=dev)
        charge = torch.empty(n_om, dtype=torch.float64, device=dev)
        portions = torch.empty((n_om, 2), dtype=torch.int32, device=dev)
        e = elements
        P = _lib.NearProblem(
            n_om, positions.data_ptr(), looks.data_ptr(), areas.data_ptr(), origins.data_ptr(),
            int(n_elements), e["start_m"].data_ptr(), e["direction"].data_ptr(),
            e["length_m"].data_ptr(), e["coefficient0"].data_ptr(),
            e["coefficient2"].data_ptr(), e["beta"].data_ptr(), e["start_ns"].data_ptr(),
            e["end_ns"].data_ptr(), radius, spectrum.data_ptr(), charge.data_ptr(),
            portions.data_ptr())
        lib = _lib.load()
        need = int(lib.lh_near_workspace_bytes(C.byref(self.struct), C.byref(P)))
        if need == 0:
            raise ValueError("invalid near-field problem (sizes, radius above the radial minimum)")
        if self._workspace is None or self._workspace.numel() < need:
            self._workspace = torch.empty(need, dtype=torch.uint8, device=dev)
        sp = _lib.stream_ptr(torch.cuda.current_stream(dev))
        _lib.check(lib.lh_near_field(C.byref(self.struct), C.byref(P), self._workspace.data_ptr(),
                                     self._workspace.numel(), sp), "lh_near_field")
        counts = portions.cpu().numpy()
        charge_h = charge.cpu().numpy()
        oms = np.flatnonzero(counts[:, 0] > 0)
        metadata = dict(radius_m=radius, table_radial_minimum_m=self.radial_minimum,
                        oms=oms.tolist(), charge_pe=[float(charge_h[om]) for om in oms],
                        elements=int(counts[:, 1].sum()), approximation=APPROXIMATION,
                        panel_m=self.panel_m, gauss_order=self.gauss_order)
        return NearField(oms, charge_h, spectrum, metadata)


def add_near_field(response, near: NearField, readout, *, mode="split-bf16", label=None):
    """Add the clamped near field to a response (``add_near_field``,
    ``near_field.py:174-217``; the shower route has no ``fine_charge_mask``, so every
    near OM takes its charge). Returns the response (changed in place)."""
    import torch
    if not len(near.oms):
        return response
    oms = near.oms
    response.charge_components_pe[oms, 2] += near.charge_pe[oms]
    active = np.asarray(response.active, bool)
    detailed = oms[active[oms]]
    omega = np.asarray(response.omega_per_ns, float)
    if len(detailed):
        rows = near.spectrum[torch.as_tensor(detailed, device=near.spectrum.device)]
        bins, _ = readout.bins(rows.to(torch.complex64), mode=mode)
        response.components_pe[detailed, :, 2] += bins.cpu().numpy().astype(float)
    spectrum = near.spectrum.cpu().numpy()
    if response.spectrum_ge2_pe is not None:
        origin = np.asarray(response.time_origin_ns, float)
        response.spectrum_ge2_pe[:, oms] += (spectrum[oms].T
                                             * np.exp(1j * omega[:, None] * origin[None, oms]))
    record = dict(near.metadata, label=label, charge_added_oms=oms.tolist(),
                  bins_added_oms=detailed.tolist())
    response.metadata.setdefault("near_field", []).append(record)
    warnings.warn(
        f"{len(oms)} OMs have source points closer than the {near.metadata['radius_m']:g} m "
        f"radial minimum of the order >=2 tables (OM index {oms.tolist()}); their order >=2 "
        f"near part uses the near-field clamp ({sum(near.metadata['charge_pe']):.3g} pe), "
        "see metadata['near_field']", RuntimeWarning, stacklevel=2)
    return response
