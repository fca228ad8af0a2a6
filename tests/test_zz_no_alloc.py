"""The flash entry point that allocates nothing, against the allocating one.

``lh_flash_transport_noalloc`` exists for callers that cannot allocate device
memory (a framework that reserves the GPU's memory up front, or a loop where
cudaMalloc would synchronise the device): it keeps its scratch in a static
device array of the library. This file is collected last so that a failure
here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# The tolerances of tests/test_flash_gpu.py for the fp32 path.
CHARGE_RTOL = 1e-3
BINS_TOL = 1e-4
WIDE_K_PAD = 208  # 78 padding columns for 65 frequencies: more padding than frequencies


@pytest.fixture(scope="module")
def plain(flash_table, flash_config):
    from lighthit_b200.flash import FlashTransport
    from lighthit_b200.model import synthetic_detector
    return FlashTransport(synthetic_detector(), flash_config, flash_table, mode="fp32")


def batch_of(pos, photons, time_ns, out, n_device=None):
    from lighthit_b200 import _lib
    return _lib.FlashBatch(
        int(pos.shape[0]), pos.data_ptr(), photons.data_ptr(), time_ns.data_ptr(),
        out["spectrum"].data_ptr(), out["components"].data_ptr(), out["charge"].data_ptr(),
        out["origin"].data_ptr(), out["active"].data_ptr(), out["status"].data_ptr(),
        n_device.data_ptr() if n_device is not None else None, 0)


def stream_ptr():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def call_noalloc(ft, pos, photons, time_ns, out, readout=None):
    from lighthit_b200 import _lib
    op = ft.readout.struct if readout is None else readout
    return _lib.load().lh_flash_transport_noalloc(
        ctypes.byref(ft.problem), ctypes.byref(op), ctypes.byref(batch_of(pos, photons, time_ns, out)),
        stream_ptr())


def wide_operator(ft):
    """The fp32 readout operator with ``WIDE_K_PAD`` columns (zeros past 2 n_omega)."""
    import torch
    from lighthit_b200 import _lib
    ro = ft.readout
    wide = torch.zeros((ro.n_bins, WIDE_K_PAD), dtype=torch.float32, device="cuda")
    wide[:, :ro.k_pad] = ro.b_fp32
    op = _lib.ReadoutOperator(ro.n_bins, WIDE_K_PAD, ro.n_tile, ro.n_tiles, wide.data_ptr(),
                              ro.b_hi.data_ptr(), ro.b_lo.data_ptr())
    return op, wide


def inputs(n, seed, golden):
    import torch
    from lighthit_b200.workloads import flash_positions
    centre = golden["om_positions_m"].mean(axis=0)
    pos_np = flash_positions(n, centre, seed=seed, om_positions=golden["om_positions_m"])
    pos = torch.tensor(pos_np, dtype=torch.float64, device="cuda")
    ph = torch.full((n,), 1e10, dtype=torch.float64, device="cuda")
    tt = torch.zeros(n, dtype=torch.float64, device="cuda")
    return pos, ph, tt


def assert_same(got, ref, rows=None):
    sl = slice(None) if rows is None else slice(0, rows)
    q_ref = ref["charge"][sl].cpu().numpy()
    q = got["charge"][sl].cpu().numpy()
    assert np.all(np.abs(q - q_ref) <= CHARGE_RTOL * np.abs(q_ref))
    c_ref = ref["components"][sl].cpu().numpy()
    c = got["components"][sl].cpu().numpy()
    assert np.isfinite(c).all()
    assert np.abs(c - c_ref).max() <= BINS_TOL * np.abs(c_ref).max()
    np.testing.assert_array_equal(got["origin"][sl].cpu().numpy(), ref["origin"][sl].cpu().numpy())
    np.testing.assert_array_equal(got["active"][sl].cpu().numpy(), ref["active"][sl].cpu().numpy())
    s_ref = ref["spectrum"][sl].cpu().numpy()
    assert np.abs(got["spectrum"][sl].cpu().numpy() - s_ref).max() <= 1e-6 * np.abs(s_ref).max()


def test_noalloc_matches_allocating_entry_point_twice(plain, flash_golden):
    """A larger call, then a smaller one: the smaller call must not pick up the
    rows the larger one left in the shared scratch, and neither call may grow
    torch's device allocation."""
    import torch
    from lighthit_b200 import _lib
    for n, seed in ((75, 202), (40, 101)):
        pos, ph, tt = inputs(n, seed, flash_golden)
        ref = plain.allocate(n)
        plain.launch(pos, ph, tt, ref, mode="fp32")
        got = plain.allocate(n)
        torch.cuda.synchronize()
        allocated, reserved = torch.cuda.memory_allocated(), torch.cuda.memory_reserved()
        assert call_noalloc(plain, pos, ph, tt, got) == _lib.LH_OK
        torch.cuda.synchronize()
        assert torch.cuda.memory_allocated() == allocated
        assert torch.cuda.memory_reserved() == reserved
        assert int(got["status"][0]) == 0
        assert_same(got, ref)


def test_noalloc_padding_wider_than_the_spectrum(plain, flash_golden):
    """A readout operator with more padding columns than frequencies, after a
    larger call filled the scratch: every padding column is rewritten."""
    import torch
    from lighthit_b200 import _lib
    op, _keep = wide_operator(plain)
    big = inputs(70, 303, flash_golden)
    assert call_noalloc(plain, *big, plain.allocate(70)) == _lib.LH_OK
    pos, ph, tt = inputs(30, 404, flash_golden)
    ref = plain.allocate(30)
    plain.launch(pos, ph, tt, ref, mode="fp32")
    got = plain.allocate(30)
    assert call_noalloc(plain, pos, ph, tt, got, readout=op) == _lib.LH_OK
    torch.cuda.synchronize()
    assert_same(got, ref)


def test_plain_rows_written_in_full(plain, flash_golden):
    """The allocating plain path on a workspace full of NaN, with the wide
    operator and a device flash count below the host count: no NaN reaches the
    outputs, and the counted flashes match the standard operator."""
    import torch
    from lighthit_b200 import _lib
    op, _keep = wide_operator(plain)
    n, counted = 24, 17
    pos, ph, tt = inputs(n, 505, flash_golden)
    ref = plain.allocate(n)
    plain.launch(pos, ph, tt, ref, mode="fp32")
    need = 2 * n * plain.n_om * WIDE_K_PAD * 4
    ws = torch.full((need // 4,), float("nan"), dtype=torch.float32, device="cuda")
    got = plain.allocate(n)
    got["components"].zero_()
    n_dev = torch.tensor([counted], dtype=torch.int32, device="cuda")
    rc = _lib.load().lh_flash_transport(
        ctypes.byref(plain.problem), ctypes.byref(op), _lib.MODES["fp32"],
        ctypes.byref(batch_of(pos, ph, tt, got, n_dev)), ctypes.c_void_p(ws.data_ptr()),
        ctypes.c_size_t(need), stream_ptr())
    assert rc == _lib.LH_OK
    torch.cuda.synchronize()
    assert np.isfinite(got["components"].cpu().numpy()).all()
    assert_same(got, ref, rows=counted)


def test_noalloc_rejects_batches_beyond_its_scratch(plain, flash_golden):
    import torch
    from lighthit_b200 import _lib
    F = 200  # 2 * 200 * 48 * 144 * 4 bytes > 4 MiB
    pos = torch.tensor(np.tile(flash_golden["flash_position_m"][:1], (F, 1)), dtype=torch.float64,
                       device="cuda")
    ph = torch.full((F,), 1e10, dtype=torch.float64, device="cuda")
    tt = torch.zeros(F, dtype=torch.float64, device="cuda")
    out = plain.allocate(F)
    assert call_noalloc(plain, pos, ph, tt, out) == _lib.LH_ESCRATCH
