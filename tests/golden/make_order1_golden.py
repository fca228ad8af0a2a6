"""Write the order-1 (grouped pencils) fixtures from the reference.

Run here (reference present):  python tests/golden/make_order1_golden.py
(after make_shower_golden.py, whose response fixture supplies the route's clock).

Workload: the README-example shower of ``make_shower_golden.setup`` with the
shower route's prompt settings (``shower/api.py:36-44``: fused bands, pixel
face 96, 192 ring nodes, cell 0.5 m). All 2000 elements emit in every band,
so the fused unit (``muon/secondary_first.py:184-204``) holds them all.

Outputs ``tests/golden/order1_c0.npz``:
* the fused unit's elements and frozen cone cosines (``prompt.py:471-481``),
  the spectral tables (``prompt.py:412-434``), acceptance monomials
  (``prompt.py:380-399``), the route's per-OM clock and the 5 ns edges;
* ``compress`` (``prompt.py:1317-1402``) of a 64-element subset: the pencil
  table (stage A);
* ``grouped_pencils_order1`` (``_prompt_numba.py:2001-2086``) of those subset
  pencils for all 48 OMs (stage B on fixed pencils), and of the pencils of
  the whole element set (stage A + B, the fine order 1 of every OM).
"""
import sys
import time
from dataclasses import replace
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from make_shower_golden import EDGES, setup  # noqa: E402
from _refenv import REPO  # noqa: E402

from lighthit import _prompt_numba as kernels  # noqa: E402
from lighthit.muon.secondary_first import _evaluation_units  # noqa: E402
from lighthit.prompt import (_element_segments, _spectral_tables, acceptance_monomials,  # noqa: E402
                             compress)
from lighthit.shower.api import ShowerConfig  # noqa: E402

PENCIL_KEYS = ("position", "direction", "w0", "w2", "time", "major", "var_major", "var_minor",
               "pos_cov")


def grouped(kernel, pencils, origins, tables, config, work, compute_bins=True):
    d = kernel.detector
    coef, ipow, jpow, degree = acceptance_monomials(kernel.acceptance()["alpha"])
    g = float(kernel.medium.g)
    y_g = (1.0 - abs(g)) / (1.0 + abs(g)) if g != 0 else 1.0
    kappa = -tables["mut"] * tables["speed"]
    eedge = np.exp(np.outer(kappa, EDGES))
    itab = kernels.interval_table(EDGES, kappa)
    return kernels.grouped_pencils_order1(
        np.ascontiguousarray(d.positions_m, float), np.ascontiguousarray(-d.orientations, float),
        np.asarray(d.effective_area_m2, float) * np.ones(len(d)), np.ascontiguousarray(origins),
        np.ascontiguousarray(work, np.int64), pencils["position"], pencils["direction"],
        pencils["w0"], pencils["w2"], pencils["time"], pencils["major"], pencils["var_major"],
        pencils["var_minor"], pencils["pos_cov"], kernels._GAUSS_TAU, kernels._GAUSS_W,
        coef, ipow, jpow, degree, g, y_g, config.path_step, config.path_step_tail,
        config.tail_exponent, tables["mus"], tables["mut"], tables["speed"], tables["s0w"],
        tables["s2w"], EDGES, eedge, itab, int(config.direct_bins), int(config.max_path_nodes),
        float(config.smoothing_factor), float(config.merge_theta_min),
        float(config.merge_theta_ratio), float(config.merge_tau_ns), float(config.merge_log_r),
        float(np.max(tables["speed"])), 1, compute_bins)


def main():
    kernel, shower, _ = setup()
    golden = REPO / "tests" / "golden"
    route = np.load(golden / "shower_c0.npz")
    origins = np.asarray(route["time_origin_ns"], float)
    prompt = ShowerConfig().prompt
    tables = _spectral_tables(kernel)
    elements = kernel._source_elements(shower)
    low, high = kernel.config.wavelength_range_nm or kernel.medium.wavelength_range_nm
    native = kernel.medium.wavelength_nm
    critical = np.r_[low, native[(native > low) & (native < high)], high]
    threshold_phase = float(np.max(kernel.medium.sample(critical)["phase_index"]))
    valid = elements.beta * threshold_phase > 1
    if not np.all(valid):
        elements = elements.subset(valid)
    band_valid = [elements.beta * phase > 1 for phase in tables["phase_index"]]
    units = _evaluation_units(tables, band_valid, True)
    fused = units[0]
    assert fused["fused"] and np.all(fused["valid"]), "every element emits in every band"
    assert not any(np.any(u["valid"]) for u in units[1:])
    subset = replace(elements, reference_phase_index=float(fused["cone"]), cone_model="frozen")
    segments = _element_segments(subset)
    config = replace(prompt, pixel_face=int(prompt.fused_pixel_face),
                     ring_nodes=int(prompt.fused_ring_nodes))
    coef, ipow, jpow, degree = acceptance_monomials(kernel.acceptance()["alpha"])
    work = np.arange(len(kernel.detector))
    out = {}
    # stage A on a subset of 64 elements, and stage B on its pencils
    pick = np.arange(0, len(subset.beta), len(subset.beta) // 64)[:64]
    small = subset.subset(np.isin(np.arange(len(subset.beta)), pick))
    small_pencils = compress(small, _element_segments(small), config)
    for k in PENCIL_KEYS:
        out[f"sub_pencil_{k}"] = small_pencils[k]
    t0 = time.perf_counter()
    q, b, groups, batches = grouped(kernel, small_pencils, origins, tables, config, work)
    print(f"subset: {len(small_pencils['w0'])} pencils, grouped {time.perf_counter() - t0:.1f} s, "
          f"{q.sum():.6f} pe, groups max {groups.max()}")
    out.update(sub_charge=q, sub_bins=b, sub_groups=groups, sub_batches=batches, sub_pick=pick)
    # stages A + B on every element
    t0 = time.perf_counter()
    pencils = compress(subset, segments, config)
    t1 = time.perf_counter()
    q, b, groups, batches = grouped(kernel, pencils, origins, tables, config, work)
    print(f"full: {len(pencils['w0'])} pencils, compress {t1 - t0:.1f} s, grouped "
          f"{time.perf_counter() - t1:.1f} s, {q.sum():.6f} pe, groups max {groups.max()}, "
          f"batches {batches.sum()}")
    out.update(full_charge=q, full_bins=b, full_groups=groups, full_batches=batches,
               full_pencils=len(pencils["w0"]), full_pencil_w0_sum=pencils["w0"].sum(),
               full_pencil_w2_sum=pencils["w2"].sum())
    names = ("start_m", "direction", "length_m", "coefficient0", "coefficient2", "beta",
             "start_ns", "end_ns")
    d = kernel.detector
    np.savez_compressed(
        golden / "order1_c0.npz", **{k: np.asarray(getattr(subset, k), float) for k in names},
        cone_cos=np.asarray(segments.cone, float), cone_phase=float(fused["cone"]),
        mus=tables["mus"], mut=tables["mut"], speed=tables["speed"], s0w=tables["s0w"],
        s2w=tables["s2w"], g=float(kernel.medium.g), coef=coef, ipow=ipow, jpow=jpow,
        degree=degree, positions_m=np.asarray(d.positions_m, float),
        looks=np.asarray(-d.orientations, float),
        areas_m2=np.asarray(d.effective_area_m2, float) * np.ones(len(d)), origins_ns=origins,
        edges_ns=EDGES, cell_m=config.cell_m, pixel_face=config.pixel_face,
        ring_nodes=config.ring_nodes, path_step=config.path_step,
        path_step_tail=config.path_step_tail, tail_exponent=config.tail_exponent,
        direct_bins=config.direct_bins, max_path_nodes=config.max_path_nodes,
        smoothing_factor=config.smoothing_factor, merge_theta_min=config.merge_theta_min,
        merge_theta_ratio=config.merge_theta_ratio, merge_tau_ns=config.merge_tau_ns,
        merge_log_r=config.merge_log_r, **out)


if __name__ == "__main__":
    main()
