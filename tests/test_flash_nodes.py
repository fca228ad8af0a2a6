"""Photons of a broadband flash at the wavelength nodes (CPU).

``flash_node_photons`` restates ``_flash_nodes`` (``transport.py:1049-1059``):
``photons * weight * shape / (weight . shape)``. The node wavelengths and
weights are the reference kernel's (``tests/golden/flash_broadband_c1.npz``).
"""
import numpy as np
import pytest

from conftest import GOLDEN


def test_node_photons_split_the_flash_by_weight_and_shape():
    from lighthit_b200.flash import flash_node_photons
    g = np.load(GOLDEN / "flash_broadband_c1.npz")
    nodes, weights = g["node_wavelength_nm"], g["node_weight_nm"]
    centre, width = float(g["shape_centre_nm"]), float(g["shape_width_nm"])

    def shape(wavelength):
        return np.exp(-((np.asarray(wavelength, float) - centre) / width) ** 2)

    photons = g["flash_photons"]
    got = flash_node_photons(nodes, weights, photons, shape)
    assert got.shape == (len(nodes), len(photons))
    assert np.allclose(got.sum(axis=0), photons, rtol=1e-14)  # the nodes share the photons
    w = weights * shape(nodes)
    assert np.allclose(got[:, 0], photons[0] * w / w.sum(), rtol=1e-15)
    with pytest.raises(ValueError):
        flash_node_photons(nodes, weights, photons, lambda x: np.zeros_like(x))
    with pytest.raises(ValueError):
        flash_node_photons(nodes, weights, photons, lambda x: -np.ones_like(x))
