"""Tables read from the reference's own objects equal the committed ones.

``ShowerTransport(kernel, data)`` with the reference's ``TransportKernel``
builds ``ShowerTables.from_reference``: the route constants, the folded order
>=2 kernels and the near-field interval read through the reference's
``ShowerTransport.tables()``. Needs the reference package and its prepared
README-configuration caches (``LIGHTHIT_REFERENCE_SRC``, ``LIGHTHIT_TABLE_WORK``
with ``shower-c0`` built by ``lighthit_b200/tables/build_tables.py``); skipped
elsewhere.
"""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import TABLES

SRC = os.environ.get("LIGHTHIT_REFERENCE_SRC")
WORK = os.environ.get("LIGHTHIT_TABLE_WORK")
pytestmark = pytest.mark.skipif(
    not (SRC and WORK and (Path(WORK) / "shower-c0" / "ge2-pack" / "pack.json").exists()),
    reason="needs the reference sources and its prepared c0 caches")


@pytest.fixture(scope="module")
def reference_route():
    if SRC not in sys.path:
        sys.path.insert(0, SRC)
    import lighthit as lh
    from lighthit.examples.synthetic import baikal_like_detector, synthetic_medium_model
    from lighthit.shower import ShowerData, ShowerTransport
    cache = Path(WORK) / "shower-c0"
    config = lh.KernelConfig(
        omega_per_ns=np.linspace(0.0, 1.2, 65), readout_omega_per_ns=np.linspace(0.0, 1.2, 321),
        relative_time_edges_ns=np.arange(-60.0, 742.5, 5.0), wavelength_nodes=3,
        scattering_degree=8, source_degree=8, azimuthal_degree=2, radial_range_m=(2.0, 150.0),
        radial_nodes=48, k_max_per_m=4.0, k_panel_per_m=0.1, k_order=6, threshold_pe=0.01,
        cache_directory=str(cache), cache_policy="require")
    kernel = lh.TransportKernel(synthetic_medium_model(), baikal_like_detector(clusters=1), config)
    route = ShowerTransport(kernel, ShowerData.of(str(cache), str(cache / "ge2-pack")))
    return route, route.tables()


def _same(built, committed):
    for key, value in committed.items():
        if key == "provenance":
            continue
        got, want = np.asarray(built[key]), np.asarray(value)
        if want.dtype.kind in "fc":
            np.testing.assert_allclose(got, want, rtol=1e-12, atol=0, err_msg=key)
        else:
            np.testing.assert_array_equal(got, want, err_msg=key)


def test_route_constants_equal_the_committed_table(reference_route):
    from lighthit_b200.tables.build_tables import route_constants
    _same(route_constants(*reference_route), dict(np.load(TABLES / "route_c0.npz")))


def test_folded_kernels_and_near_interval_equal_the_committed_tables(reference_route):
    from lighthit_b200.tables.build_tables import folded_kernels, near_interval
    _same(folded_kernels(*reference_route), dict(np.load(TABLES / "ge2_fold_48om_2-150m.npz")))
    _same(near_interval(*reference_route), dict(np.load(TABLES / "near_c0.npz")))


def test_response_class_is_the_reference_class(reference_route):
    from lighthit.transport import HybridTransportResponse
    from lighthit_b200.shower import response_class
    assert response_class() is HybridTransportResponse
