"""The reference's on-disk table formats, read without the reference installed.

The reference writes its prepared tables once and reads them on every run;
the device route reads the same files:

* ``folded.npy`` + ``folded.json`` (``save_folded`` / ``load_folded``,
  ``band_fold.py:219-242``, format ``lighthit/ge2-band-fold/1``): the
  band-folded order >=2 bundle a ``ShowerData.ge2_band_fold`` directory holds.
  :func:`load_folded_pack` returns the dict :class:`~lighthit_b200.shower.ShowerTables`
  and :class:`~lighthit_b200.ge2.Ge2Table` take.
* ``pack.json`` + ``<n>.npy`` (``Ge2KernelStore.save`` / ``load``,
  ``shower_basis.py:317-349``, schema ``lighthit/ge2-kernel-pack/1``): the
  per-wavelength order >=2 bundles of ``ShowerData.ge2_pack``.
  :func:`load_kernel_pack` returns them by key; :func:`near_table` cuts a
  bundle's first radial interval for the near-field clamp
  (:class:`~lighthit_b200.near.NearTable`).
* ``transport-<key>.npz`` (``ResponseCache.save`` / ``load``,
  ``cache.py:485-507``): one wavelength's multipole response cache.
  :func:`load_response_cache` returns the flash path's
  :class:`~lighthit_b200.flash.FlashTable`.

The readers check the format tags the reference writes and raise its
``ValueError`` for a foreign pack.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

__all__ = ["FOLD_FORMAT", "PACK_SCHEMA", "load_folded_pack", "load_kernel_pack",
           "frequency_indices", "near_table", "load_response_cache"]

FOLD_FORMAT = "lighthit/ge2-band-fold/1"   # band_fold.py:47
PACK_SCHEMA = "lighthit/ge2-kernel-pack/1"  # shower_basis.py:25
MOMENT_ORDERS = ("one_finite_L", "two_or_more")  # cache.py:65, the cached orders


def _typed(meta):
    """The array fields of a bundle's metadata as the reference types them."""
    out = dict(meta)
    for key in ("pair_lambda", "pair_mu"):
        if key in out:
            out[key] = np.asarray(out[key], np.int64)
    for key in ("omega", "log_r", "absorption", "speed"):
        if key in out:
            out[key] = np.asarray(out[key], float)
    return out


def load_folded_pack(directory, *, mmap=False):
    """``load_folded`` (``band_fold.py:229-242``): the folded bundle of a
    ``folded.npy`` + ``folded.json`` directory, with ``bands`` (the node bands
    of its fold) lifted out of the fold metadata."""
    directory = Path(directory)
    meta = json.loads((directory / "folded.json").read_text())
    if meta.pop("format", None) != FOLD_FORMAT:
        raise ValueError(f"{directory} is not a {FOLD_FORMAT} pack")
    out = _typed(meta)
    out["coefficients"] = np.load(directory / "folded.npy", mmap_mode="r" if mmap else None)
    if out.get("phase") != "flight":
        raise ValueError("the device route needs flight-phase folded kernels")
    fold = out.get("band_fold") or {}
    if "bands" in fold:
        out["bands"] = np.asarray(fold["bands"], np.int64)
    return out


def load_kernel_pack(directory, *, mmap=False):
    """``Ge2KernelStore.load`` (``shower_basis.py:331-349``): ``{key: bundle}``
    with the reference's key (``shower_basis.py:176-179``): the directional
    table name of every kernel wavelength, the source degree and the frequency
    indices of the bundle."""
    directory = Path(directory)
    header = json.loads((directory / "pack.json").read_text())
    if header.get("schema") != PACK_SCHEMA:
        raise ValueError("unsupported order >=2 kernel pack")
    bundles = {}
    for item in header["bundles"]:
        meta = _typed(item["meta"])
        key = (tuple(item["key"][0]), int(item["key"][1]), tuple(item["key"][2]))
        meta["coefficients"] = np.load(directory / item["file"],
                                       mmap_mode="r" if mmap else None)
        bundles[key] = meta
    return bundles


def frequency_indices(n_grid, frequency_nodes):
    """``_frequency_indices`` (``shower_basis.py:352-362``): the cache frequencies
    a route of ``frequency_nodes`` nodes takes from a grid of ``n_grid``."""
    if not 4 <= int(frequency_nodes) <= int(n_grid):
        raise ValueError("frequency_nodes must lie between 4 and the cache grid size")
    idx = np.unique(np.rint(np.linspace(0, n_grid - 1, int(frequency_nodes))).astype(int))
    if len(idx) != int(frequency_nodes):
        raise ValueError("frequency_nodes exceed distinct cache frequencies")
    return idx


def near_table(bundle, indices=None):
    """The near-field table of one per-wavelength bundle: radial interval 0 of
    every wavelength's spline at the route's frequencies (the only part the
    clamp of ``near_field.py:91-171`` reads: every point closer than the radial
    minimum takes the amplitude there)."""
    if bundle.get("phase") != "flight":
        raise ValueError("near-field table needs flight-phase splines")
    coef = np.asarray(bundle["coefficients"])
    omega = np.asarray(bundle["omega"], float)
    if indices is not None:
        coef, omega = coef[..., indices], omega[indices]
    log_r = np.asarray(bundle["log_r"], float)
    return dict(coefficients=np.ascontiguousarray(coef[:, 0], np.complex64), log_r=log_r[:2],
                radial_high_m=float(np.exp(log_r[-1])), omega=omega,
                absorption=np.asarray(bundle["absorption"], float),
                speed=np.asarray(bundle["speed"], float), degree=int(bundle["degree"]),
                acceptance_degree=int(bundle["acceptance_degree"]),
                pair_lambda=np.asarray(bundle["pair_lambda"], np.int64),
                pair_mu=np.asarray(bundle["pair_mu"], np.int64))


def load_response_cache(path):
    """``ResponseCache.load`` (``cache.py:500-507``) as the flash path's table:
    the radii, frequencies and scattering moments of one wavelength with its
    medium, spatial degree and radial phase convention."""
    from .flash import FlashTable
    from .model import Medium
    with np.load(path, allow_pickle=False) as data:
        meta = json.loads(str(data["metadata"]))
        if tuple(meta.get("moment_orders", MOMENT_ORDERS)) != MOMENT_ORDERS:
            raise ValueError("Unsupported cached scattering-order convention")
        m = meta["medium"]
        medium = Medium(float(m["absorption_per_m"]), float(m["scattering_per_m"]),
                        float(m["g"]), float(m["group_index"]),
                        float(m.get("wavelength_nm", 450.0)))
        return FlashTable(np.asarray(data["omega_per_ns"], float),
                          np.asarray(data["radii_m"], float), np.asarray(data["moments"]),
                          medium, str(meta.get("radial_phase", "none")),
                          int(meta["settings"]["spatial_degree"]))
