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


@pytest.fixture(scope="module")
def plain(flash_table, flash_config):
    from lighthit_b200.flash import FlashTransport
    from lighthit_b200.model import synthetic_detector
    return FlashTransport(synthetic_detector(), flash_config, flash_table, mode="fp32")


def call_noalloc(ft, pos, photons, time_ns, out):
    import torch
    from lighthit_b200 import _lib
    lib = _lib.load()
    batch = _lib.FlashBatch(
        int(pos.shape[0]), pos.data_ptr(), photons.data_ptr(), time_ns.data_ptr(),
        out["spectrum"].data_ptr(), out["components"].data_ptr(), out["charge"].data_ptr(),
        out["origin"].data_ptr(), out["active"].data_ptr(), out["status"].data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib.lh_flash_transport_noalloc(ctypes.byref(ft.problem), ctypes.byref(ft.readout.struct),
                                          ctypes.byref(batch), stream)


def test_noalloc_matches_allocating_entry_point_twice(plain, flash_golden):
    import torch
    from lighthit_b200 import _lib
    from lighthit_b200.workloads import flash_positions
    centre = flash_golden["om_positions_m"].mean(axis=0)
    draws = [flash_positions(n, centre, seed=s, om_positions=flash_golden["om_positions_m"])
             for n, s in ((40, 101), (75, 202))]
    for pos_np in draws:  # two calls in a row share (and reuse) the static scratch
        F = len(pos_np)
        pos = torch.tensor(pos_np, dtype=torch.float64, device="cuda")
        ph = torch.full((F,), 1e10, dtype=torch.float64, device="cuda")
        tt = torch.zeros(F, dtype=torch.float64, device="cuda")
        ref = plain.allocate(F)
        plain.launch(pos, ph, tt, ref, mode="fp32")
        got = plain.allocate(F)
        assert call_noalloc(plain, pos, ph, tt, got) == _lib.LH_OK
        torch.cuda.synchronize()
        assert int(got["status"][0]) == 0
        q_ref = ref["charge"].cpu().numpy()
        q = got["charge"].cpu().numpy()
        assert np.all(np.abs(q - q_ref) <= CHARGE_RTOL * np.abs(q_ref))
        c_ref = ref["components"].cpu().numpy()
        c = got["components"].cpu().numpy()
        assert np.abs(c - c_ref).max() <= BINS_TOL * np.abs(c_ref).max()
        np.testing.assert_array_equal(got["origin"].cpu().numpy(), ref["origin"].cpu().numpy())
        np.testing.assert_array_equal(got["active"].cpu().numpy(), ref["active"].cpu().numpy())
        s_ref = ref["spectrum"].cpu().numpy()
        assert np.abs(got["spectrum"].cpu().numpy() - s_ref).max() <= 1e-6 * np.abs(s_ref).max()


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
