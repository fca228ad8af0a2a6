"""The oracle reproduces the reference's own float64 outputs (fixtures)."""
import numpy as np
import pytest

from conftest import GOLDEN, TABLES, oracle_config, oracle_detector
from oracle.flash import transport_flash
from oracle.readout import readout_bins


def test_readout_oracle_matches_reference():
    g = np.load(GOLDEN / "readout_c0.npz")
    bins = readout_bins(g["omega_per_ns"], g["relative"], g["edges_ns"], g["readout_omega_per_ns"])
    assert np.max(np.abs(bins - g["bins"])) < 1e-13


def test_flash_oracle_matches_reference(flash_golden):
    g = flash_golden
    table = dict(np.load(TABLES / "flash_450nm_2-250m.npz"))
    for i in range(len(g["flash_photons"])):
        r = transport_flash(table, oracle_detector(g),
                            dict(position_m=g["flash_position_m"][i], photons=g["flash_photons"][i],
                                 time_ns=g["flash_time_ns"][i]), oracle_config(g))
        q = g["charge_components_pe"][i]
        assert np.max(np.abs(r["charge_components_pe"] - q) / np.maximum(np.abs(q), 1e-300)) < 1e-12
        ref = g["components_pe"][i]
        assert np.max(np.abs(r["components_pe"] - ref)) <= 1e-6 * max(np.abs(ref).max(), 1e-30)
        np.testing.assert_array_equal(r["active"], g["active"][i])
        np.testing.assert_array_equal(r["time_origin_ns"], g["time_origin_ns"][i])
        spec = g["spectrum_pe"][i]
        assert np.max(np.abs(r["spectrum_pe"] - spec)) <= 1e-6 * np.abs(spec).max()


def test_flash_oracle_raises_like_reference(flash_golden):
    g = flash_golden
    table = dict(np.load(TABLES / "flash_450nm_2-250m.npz"))
    with pytest.raises(ValueError, match="outside radial_range_m"):
        transport_flash(table, oracle_detector(g),
                        dict(position_m=g["raise_position_m"], photons=1e10, time_ns=0.0),
                        oracle_config(g))
    assert "outside radial_range_m" in str(g["raise_message"])
