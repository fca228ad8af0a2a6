"""Device flash path vs the reference's float64 outputs (fixtures) and the oracle."""
import numpy as np
import pytest

from conftest import TABLES, oracle_config, oracle_detector

pytestmark = pytest.mark.gpu

# Per-OM charge: relative to the reference, OMs with q >= threshold (north-star bar 1e-3).
CHARGE_RTOL = 1e-3
# Fourier-inverted bins (orders 1, 2): max error over an OM's bins relative to the
# largest bin of that flash and order.
BINS_TOL = {"fp32": 1e-4, "split-bf16": 1e-4, "bf16": 3e-2}


@pytest.fixture(scope="module")
def transports(flash_table, flash_config):
    from lighthit_b200.flash import FlashTransport
    from lighthit_b200.model import synthetic_detector
    det = synthetic_detector()
    return {m: FlashTransport(det, flash_config, flash_table, mode=m) for m in BINS_TOL}


def golden_batch(g):
    keep = np.arange(len(g["flash_photons"]))
    return g["flash_position_m"][keep], g["flash_photons"][keep], g["flash_time_ns"][keep]


@pytest.mark.parametrize("mode", list(BINS_TOL))
def test_flash_batch_matches_reference(transports, flash_golden, mode):
    g = flash_golden
    ft = transports[mode]
    pos, ph, t = golden_batch(g)
    out = ft.run(pos, ph, t)
    charge = out["charge"].cpu().numpy()
    comps = out["components"].cpu().numpy().transpose(0, 1, 3, 2)  # (F, D, bins, 3)
    spec = out["spectrum"].cpu().numpy().transpose(0, 2, 1, 3)    # (F, w, D, 3)
    origin = out["origin"].cpu().numpy()
    active = out["active"].cpu().numpy()
    thr = float(g["threshold_pe"])
    for i in range(len(ph)):
        q_ref = g["charge_components_pe"][i]
        tot_ref = q_ref.sum(axis=1)
        sel = tot_ref >= thr
        rel = np.abs(charge[i].sum(axis=1) - tot_ref) / np.maximum(np.abs(tot_ref), 1e-300)
        assert rel[sel].max(initial=0) < CHARGE_RTOL, (i, rel.max())
        for o in range(3):
            err = np.abs(charge[i, :, o] - q_ref[:, o])
            assert np.all(err <= CHARGE_RTOL * np.abs(q_ref[:, o]) + 1e-6 * np.abs(tot_ref)), (i, o)
        # clocks are float64 geometry: bit-identical
        np.testing.assert_array_equal(origin[i], g["time_origin_ns"][i])
        # active identical except within tolerance of the threshold
        near = np.abs(tot_ref - thr) <= CHARGE_RTOL * thr
        a = (active[i] & 1).astype(bool)
        assert np.array_equal(a[~near], g["active"][i][~near]), i
        assert not np.any(active[i] & 6)
        ref_c = g["components_pe"][i]
        # order 0: same bin index (bit-exact assignment), value to float32 precision
        np.testing.assert_array_equal(comps[i, :, :, 0] != 0, ref_c[:, :, 0] != 0)
        assert np.allclose(comps[i, :, :, 0], ref_c[:, :, 0], rtol=1e-5, atol=0)
        for o in (1, 2):
            scale = max(np.abs(ref_c[:, :, o]).max(), 1e-30)
            assert np.abs(comps[i, :, :, o] - ref_c[:, :, o]).max() <= BINS_TOL[mode] * scale, (i, o)
        ref_s = g["spectrum_pe"][i]
        assert np.abs(spec[i] - ref_s).max() <= 1e-4 * np.abs(ref_s).max(), i


def test_flash_alone_equals_in_batch(transports, flash_golden):
    ft = transports["split-bf16"]
    pos, ph, t = golden_batch(flash_golden)
    batch = ft.run(pos, ph, t)
    for i in (0, 5, len(ph) - 1):
        alone = ft.run(pos[i:i + 1], ph[i:i + 1], t[i:i + 1])
        for key in ("spectrum", "components", "charge", "origin", "active"):
            assert np.array_equal(alone[key][0].cpu().numpy(), batch[key][i].cpu().numpy()), key


def test_flash_drop_in_transport_and_errors(transports, flash_golden):
    from lighthit_b200.model import IsotropicFlash
    g = flash_golden
    ft = transports["split-bf16"]
    r = ft.transport(IsotropicFlash.monochromatic(g["flash_position_m"][0], 1e10, 450.0))
    assert r.spectrum_pe.shape == (65, 48, 3) and r.components_pe.shape == (48, 160, 3)
    ref = g["charge_components_pe"][0].sum(axis=1)
    assert np.max(np.abs(r.charge_pe - ref) / ref) < CHARGE_RTOL
    with pytest.raises(ValueError, match="outside radial_range_m"):
        ft.transport(IsotropicFlash.monochromatic(g["raise_position_m"], 1e10, 450.0))
    with pytest.raises(ValueError, match="coincide"):
        ft.transport(IsotropicFlash.monochromatic(g["om_positions_m"][3], 1e10, 450.0))


def test_flash_against_oracle_fresh_positions(transports, flash_table):
    """Flashes beyond the fixture set, checked against the oracle on the CPU."""
    from lighthit_b200.workloads import flash_positions
    from oracle.flash import transport_flash
    g = np.load(TABLES.parent.parent / "tests" / "golden" / "flash_c1.npz")
    table = dict(np.load(TABLES / "flash_450nm_2-250m.npz"))
    ft = transports["split-bf16"]
    centre = g["om_positions_m"].mean(axis=0)
    pos = flash_positions(40, centre, seed=99, om_positions=g["om_positions_m"])
    out = ft.run(pos, 1e10)
    charge = out["charge"].cpu().numpy()
    comps = out["components"].cpu().numpy()
    for i in range(0, 40, 7):
        r = transport_flash(table, oracle_detector(g), dict(position_m=pos[i], photons=1e10,
                                                            time_ns=0.0), oracle_config(g))
        q = r["charge_components_pe"].sum(axis=1)
        assert np.max(np.abs(charge[i].sum(axis=1) - q) / q) < CHARGE_RTOL
        c = comps[i].transpose(0, 2, 1)
        for o in (1, 2):
            assert (np.abs(c[:, :, o] - r["components_pe"][:, :, o]).max()
                    <= 1e-4 * np.abs(r["components_pe"][:, :, o]).max())
