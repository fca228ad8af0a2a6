"""The reference's on-disk table formats read by ``lighthit_b200.formats``.

The files under ``tests/golden/formats/`` were written by the reference's own
writers (``make_formats_golden.py``: ``band_fold.save_folded``,
``Ge2KernelStore.save``, ``ResponseCache.save``) from slices of the committed
tables; these tests rebuild the slices and check that the readers return them.
"""
import json
import shutil

import numpy as np
import pytest

from conftest import GOLDEN, TABLES

FORMATS = GOLDEN / "formats"
N_INT, N_OMEGA = 2, 4
PACK_INDICES = ((0, 16, 32, 64), (0, 1, 2, 3))


def test_folded_pack_reads_as_the_route_table():
    from lighthit_b200.formats import load_folded_pack
    got = load_folded_pack(FORMATS / "folded")
    t = np.load(TABLES / "ge2_fold_48om_2-150m.npz")
    np.testing.assert_array_equal(got["coefficients"], t["coefficients"][:, :N_INT, ..., :N_OMEGA])
    assert got["coefficients"].dtype == np.complex64
    np.testing.assert_array_equal(got["log_r"], t["log_r"][:N_INT + 1])
    np.testing.assert_array_equal(got["omega"], t["omega"][:N_OMEGA])
    for key in ("absorption", "speed", "pair_lambda", "pair_mu", "bands"):
        np.testing.assert_array_equal(got[key], t[key])
    assert got["degree"] == int(t["degree"]) and got["phase"] == "flight"
    assert got["pair_lambda"].dtype == np.int64


def test_folded_pack_feeds_the_device_table_builder():
    """The read bundle has every field ``Ge2Table`` takes (checked on the host:
    the table's constructor derives its channel layout from them)."""
    from lighthit_b200.formats import load_folded_pack
    got = load_folded_pack(FORMATS / "folded")
    for key in ("coefficients", "degree", "acceptance_degree", "omega", "pair_lambda",
                "pair_mu", "log_r", "phase", "absorption", "speed"):
        assert key in got, key


def test_foreign_folded_pack_is_refused(tmp_path):
    from lighthit_b200.formats import load_folded_pack
    shutil.copytree(FORMATS / "folded", tmp_path / "folded")
    meta = json.loads((tmp_path / "folded" / "folded.json").read_text())
    meta["format"] = "something/else"
    (tmp_path / "folded" / "folded.json").write_text(json.dumps(meta))
    with pytest.raises(ValueError, match="is not a lighthit/ge2-band-fold/1 pack"):
        load_folded_pack(tmp_path / "folded")


def test_kernel_pack_bundles_and_near_table():
    from lighthit_b200.formats import load_kernel_pack, near_table
    bundles = load_kernel_pack(FORMATS / "pack")
    n = np.load(TABLES / "near_c0.npz")
    rng = np.random.default_rng(5)
    assert len(bundles) == len(PACK_INDICES)
    for b, indices in enumerate(PACK_INDICES):
        shape = (3, N_INT, int(n["degree"]) + 1, len(n["pair_lambda"]), 4, N_OMEGA)
        coef = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
        key = ((f"table-{b}-a", f"table-{b}-b", f"table-{b}-c"), 8, indices)
        got = bundles[key]
        np.testing.assert_array_equal(got["coefficients"], coef)
        np.testing.assert_array_equal(got["omega"], n["omega"][list(indices)])
        near = near_table(got)
        np.testing.assert_array_equal(near["coefficients"], coef[:, 0])
        np.testing.assert_array_equal(near["log_r"], got["log_r"][:2])
        assert near["radial_high_m"] == pytest.approx(150.0, rel=1e-12)
        part = near_table(got, [0, 2])
        np.testing.assert_array_equal(part["coefficients"], coef[:, 0][..., [0, 2]])


def test_frequency_indices_match_the_reference_rule():
    from lighthit_b200.formats import frequency_indices
    np.testing.assert_array_equal(frequency_indices(65, 65), np.arange(65))
    np.testing.assert_array_equal(frequency_indices(65, 5), [0, 16, 32, 48, 64])
    with pytest.raises(ValueError):
        frequency_indices(65, 3)


def test_response_cache_reads_as_the_flash_table():
    from lighthit_b200.formats import load_response_cache
    table = load_response_cache(FORMATS / "transport-450.npz")
    f = np.load(TABLES / "flash_450nm_2-250m.npz")
    np.testing.assert_array_equal(table.radii_m, f["radii_m"][:6])
    np.testing.assert_array_equal(table.omega_per_ns, f["omega_per_ns"][:5])
    np.testing.assert_array_equal(table.moments, f["moments"][:5, :6])
    assert table.degree == int(f["degree"]) and table.radial_phase == str(f["radial_phase"])
    assert table.medium.absorption_per_m == float(f["absorption_per_m"])
    assert table.medium.group_index == float(f["group_index"])
    assert table.medium.wavelength_nm == float(f["wavelength_nm"])


def test_flash_table_from_cache_file():
    from lighthit_b200.flash import FlashTable
    table = FlashTable.from_cache_file(FORMATS / "transport-450.npz")
    f = np.load(TABLES / "flash_450nm_2-250m.npz")
    np.testing.assert_array_equal(table.moments, f["moments"][:5, :6])


@pytest.mark.gpu
def test_route_on_tables_read_from_packs_equals_the_route(tmp_path):
    """The README shower on tables read from a full-size folded pack (in the
    format the readers above are pinned to) equals the route on the committed
    tables (up to the run-to-run rounding of the order-1 float64 atomics)."""
    from lighthit_b200.formats import FOLD_FORMAT
    from lighthit_b200.shower import ShowerTables, ShowerTransport
    t = dict(np.load(TABLES / "ge2_fold_48om_2-150m.npz"))
    pack = tmp_path / "folded"
    pack.mkdir()
    np.save(pack / "folded.npy", t["coefficients"])
    meta = {k: (np.asarray(v).tolist() if np.ndim(v) else np.asarray(v).item())
            for k, v in t.items() if k not in ("coefficients", "bands", "scale", "provenance")}
    meta["band_fold"] = {"bands": t["bands"].tolist(), "rank": len(t["bands"])}
    (pack / "folded.json").write_text(json.dumps(dict(format=FOLD_FORMAT, **meta)))
    e = np.load(GOLDEN / "order0_c0.npz")
    el = {k: np.array(e[k]) for k in ("start_m", "direction", "length_m", "coefficient0",
                                      "coefficient2", "beta", "start_ns", "end_ns")}
    ref = ShowerTransport(ShowerTables.synthetic("c0"))(el)
    got = ShowerTransport(ShowerTables.from_packs(TABLES / "route_c0.npz", pack,
                                                  near=TABLES / "near_c0.npz"))(el)
    scale = np.abs(ref.charge_pe).max()
    assert np.abs(got.charge_components_pe - ref.charge_components_pe).max() <= 1e-10 * scale
    assert np.abs(got.components_pe - ref.components_pe).max() <= 1e-10 * scale
    np.testing.assert_array_equal(got.active, ref.active)
    np.testing.assert_array_equal(got.time_origin_ns, ref.time_origin_ns)
