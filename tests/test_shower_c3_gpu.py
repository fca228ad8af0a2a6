"""Config 3 (high-resolution precision study): the device route against the
reference's float64 ``ShowerTransport`` with each readout precision (``-m gpu``).

384 OMs, 1-300 m tables with 96 radial nodes, 8 wavelength nodes folded to 3
node bands, scattering/source degree 16, azimuthal degree 4 (133 source
channels), 1025 readout nodes, 1 ns bins from -60 to 2000 ns (2060 bins).
Fixture: ``tests/golden/shower_c3.npz`` (``make_shower_c3_golden.py``): the
first 12 showers of the seeded config-3 stream (20000 elements each). Shower 11
makes the reference's control-variate order 0 raise (its disk quadrature does
not converge); the reference's direct ray form, which the device evaluates,
converges there, so that shower is checked against the CPU oracle's whole route
(``shower_c3_oracle.npz``, ``make_shower_c3_oracle.py``: the ray form with the
reference's adaptive order doubling). The showers of a mode run as one
stage-major batch.

The >=2 contraction of the full spectra and the readout run in the mode
under study: FP32 on the CUDA cores, or on the tensor cores with split-BF16
(hi + lo, three products, FP32 accumulate) or BF16 (one product). Order 0 and
1 charges do not depend on it (the >=2 charge is the exact zero-frequency
contraction, always FP32); bins, spectra and the per-order errors against the
reference are reported per mode. Bars: charge as for
the other configs; bins L1 per order BINS_L1[mode] of the OM's charge and
spectrum SPECTRUM[mode] of each OM's largest value. FP32 and split-BF16 (three
BF16 parts per operand in the contraction, two in the readout) keep the >=2
bins within 1e-3. A single BF16 product (8 significant bits per operand) in
both the contraction and the readout leaves ~0.7 of the OM's charge as bins
L1 and ~16 % spectrum error on the order >=2 waveforms of this window (2060
bins, 130 terms per bin that largely cancel): the study's answer is that BF16
alone is not usable here, which is why the route contracts and reads out in
split-BF16; its bars only bound that measured error.
"""
import numpy as np
import pytest

from conftest import GOLDEN

ORDER0, ORDER1, ORDER2 = 1e-4, 1e-5, 1e-4
BINS_L1 = {"fp32": 1e-3, "split-bf16": 1e-3, "bf16": 1.0}
SPECTRUM = {"fp32": 1e-3, "split-bf16": 1e-3, "bf16": 0.25}
N_SHOWERS = 12

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stream():
    from lighthit_b200.shower import ShowerTables
    from lighthit_b200.workloads import gaussian_shower, shower_stream
    g = np.load(GOLDEN / "shower_c3.npz")
    tables = ShowerTables.synthetic("c3")
    poses = shower_stream(N_SHOWERS, tables.positions.mean(axis=0), seed=31,
                          low_elements=20000, high_elements=20000)
    kept, sources = [], []
    for k, s in enumerate(poses):
        el = gaussian_shower(s["position_m"], s["direction"],
                             charged_track_length_m=s["charged_track_length_m"],
                             elements=s["elements"], seed=s["seed"])
        assert float(el["start_m"].sum() + el["start_ns"].sum()) == float(g[f"s{k}_checksum"])
        kept.append(k)
        sources.append(el)
    return tables, merged(g), kept, sources


def merged(g):
    """The reference's fixture with the oracle's response for the shower the
    reference rejects."""
    out = dict(g)
    oracle = np.load(GOLDEN / "shower_c3_oracle.npz")
    for k in range(N_SHOWERS):
        if f"s{k}_raises" in g.files:
            assert float(oracle[f"s{k}_checksum"]) == float(g[f"s{k}_checksum"])
            for key in ("charge", "active", "origin", "active_ids", "components", "level",
                        "spectrum"):
                out[f"s{k}_{key}"] = oracle[f"s{k}_{key}"]
    return out


@pytest.fixture(scope="module", params=["split-bf16", "fp32", "bf16"])
def routed(request, stream):
    from dataclasses import replace
    from lighthit_b200.shower import ShowerTransport
    tables, g, kept, sources = stream
    route = ShowerTransport(tables, config=replace(tables.settings, readout_mode=request.param,
                                                   contraction_mode=request.param))
    return request.param, route.batch(sources), g, kept, tables.threshold


def test_clocks_and_active(routed):
    _, responses, g, kept, threshold = routed
    for k, r in zip(kept, responses):
        assert np.array_equal(r.time_origin_ns, g[f"s{k}_origin"]), k
        ref = g[f"s{k}_active"]
        total = g[f"s{k}_charge"].sum(axis=1)
        near = np.abs(total - threshold) <= ORDER2 * np.maximum(np.abs(total), threshold)
        assert np.array_equal(r.active[~near], ref[~near]), k
        assert np.array_equal(np.asarray(r.metadata["ge2_charge_level"]), g[f"s{k}_level"]), k


def test_charge_per_order(routed):
    mode, responses, g, kept, threshold = routed
    worst = np.zeros(3)
    for k, r in zip(kept, responses):
        ref = g[f"s{k}_charge"]
        got = r.charge_components_pe
        total = ref.sum(axis=1)
        big = total >= threshold
        if not big.any():
            continue
        for order, tol in enumerate((ORDER0, ORDER1, ORDER2)):
            scale = np.abs(ref[big, order]) if order < 2 else np.abs(total[big])
            err = np.abs(got[big, order] - ref[big, order]) / np.maximum(scale, 1e-300)
            if order < 2:
                err = err[ref[big, order] > 1e-3 * total[big]]
            worst[order] = max(worst[order], err.max(initial=0.0))
            assert err.max(initial=0.0) <= tol, (k, order, err.max())
    print(f"\nc3 {mode}: worst per-order relative charge error {worst}")


def test_bins_and_spectrum(routed):
    mode, responses, g, kept, _ = routed
    worst = np.zeros(3)
    spec_worst = 0.0
    for k, r in zip(kept, responses):
        ids = g[f"s{k}_active_ids"]
        if not len(ids):
            continue
        both = ids[r.active[ids]]
        pos = np.searchsorted(ids, both)
        ref = g[f"s{k}_components"][pos].astype(float)
        got = r.components_pe[both]
        charge = np.maximum(np.abs(g[f"s{k}_charge"][both]).sum(axis=1), 1e-300)
        for order in range(3):
            l1 = np.abs(got[:, :, order] - ref[:, :, order]).sum(axis=1) / charge
            worst[order] = max(worst[order], l1.max())
        spec_ref = g[f"s{k}_spectrum"][:, pos]
        scale = np.abs(spec_ref).max(axis=0)
        spec = np.abs(r.spectrum_ge2_pe[:, both] - spec_ref).max(axis=0) / scale
        spec_worst = max(spec_worst, spec.max())
    print(f"\nc3 {mode}: worst per-order bins L1 / charge {worst}, spectrum {spec_worst:.2e}")
    assert worst.max() <= BINS_L1[mode], (mode, worst)
    assert spec_worst < SPECTRUM[mode], (mode, spec_worst)
