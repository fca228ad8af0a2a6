"""Broadband flashes on the device against the reference (``-m gpu``).

Fixture: ``tests/golden/flash_broadband_c1.npz`` (``make_flash_broadband_golden.py``):
``TransportKernel.transport(IsotropicFlash.broadband(...))`` of nine flashes of
the seed-11 workload with a Gaussian spectral shape, transported by the
reference at its three wavelength nodes (``transport.py:1049-1164``). Here one
fused launch per node (that node's table, the common clock of the fastest
node) and ``lh_flash_combine`` (sum, mask, range check). Bars as for the
monochromatic flashes: per-OM charge 1e-3, bins 1e-4 of the largest bin,
clocks bit-identical.
"""
import numpy as np
import pytest

from conftest import TABLES

pytestmark = pytest.mark.gpu

CHARGE_RTOL = 1e-3
BINS_TOL = 1e-4


@pytest.fixture(scope="module")
def broadband(flash_config):
    from conftest import GOLDEN
    from lighthit_b200.flash import BroadbandFlashTransport, FlashTable
    from lighthit_b200.model import synthetic_detector
    g = np.load(GOLDEN / "flash_broadband_c1.npz")
    nodes = g["node_wavelength_nm"]
    names = ["flash_450nm_2-250m.npz" if abs(w - 450.0) < 1e-9 else f"flash_{w:.2f}nm_2-250m.npz"
             for w in nodes]
    tables = [FlashTable.load(TABLES / n) for n in names]
    bt = BroadbandFlashTransport(synthetic_detector(), flash_config, tables, nodes,
                                 g["node_weight_nm"], mode="split-bf16")
    centre, width = float(g["shape_centre_nm"]), float(g["shape_width_nm"])

    def shape(wavelength_nm):
        return np.exp(-((np.asarray(wavelength_nm, float) - centre) / width) ** 2)

    return bt, g, shape


def test_broadband_batch_matches_reference(broadband):
    bt, g, shape = broadband
    out = bt.run(g["flash_position_m"], g["flash_photons"], g["flash_time_ns"], shape)
    charge = out["charge"].cpu().numpy()
    comps = out["components"].cpu().numpy().transpose(0, 1, 3, 2)
    spec = out["spectrum"].cpu().numpy().transpose(0, 2, 1, 3)
    origin = out["origin"].cpu().numpy()
    active = out["active"].cpu().numpy()
    thr = 0.01
    for i in range(len(g["flash_photons"])):
        ref = g["charge_components_pe"][i]
        tot = ref.sum(axis=1)
        rel = np.abs(charge[i].sum(axis=1) - tot) / np.maximum(np.abs(tot), 1e-300)
        assert rel[tot >= thr].max(initial=0) < CHARGE_RTOL, (i, rel.max())
        np.testing.assert_array_equal(origin[i], g["time_origin_ns"][i])
        near = np.abs(tot - thr) <= CHARGE_RTOL * thr
        assert np.array_equal((active[i] & 1).astype(bool)[~near], g["active"][i][~near]), i
        assert not np.any(active[i] & 6)
        ref_c = g["components_pe"][i]
        np.testing.assert_array_equal(comps[i, :, :, 0] != 0, ref_c[:, :, 0] != 0)
        assert np.allclose(comps[i, :, :, 0], ref_c[:, :, 0], rtol=1e-5, atol=0)
        for o in (1, 2):
            scale = max(np.abs(ref_c[:, :, o]).max(), 1e-30)
            assert np.abs(comps[i, :, :, o] - ref_c[:, :, o]).max() <= BINS_TOL * scale, (i, o)
        ref_s = g["spectrum_pe"][i]
        assert np.abs(spec[i] - ref_s).max() <= 1e-4 * np.abs(ref_s).max(), i


def test_broadband_drop_in_transport(broadband):
    from lighthit_b200.model import IsotropicFlash
    bt, g, shape = broadband
    i = len(g["flash_photons"]) - 1
    r = bt.transport(IsotropicFlash.broadband(g["flash_position_m"][i], float(g["flash_photons"][i]),
                                              shape, time_ns=float(g["flash_time_ns"][i])))
    assert r.metadata["wavelength_nm"] == pytest.approx(list(g["node_wavelength_nm"]))
    np.testing.assert_array_equal(r.time_origin_ns, g["time_origin_ns"][i])
    tot = g["charge_components_pe"][i].sum(axis=1)
    big = tot >= 0.01
    assert np.all(np.abs(r.charge_pe[big] - tot[big]) <= CHARGE_RTOL * np.abs(tot[big]))
    with pytest.raises(ValueError):
        bt.transport(IsotropicFlash.monochromatic(g["flash_position_m"][0], 1e10, 450.0))
