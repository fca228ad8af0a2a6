"""Failure detection on the device without a fault (``-m gpu``).

Every wait of the tensor-core kernels on an mbarrier is bounded in time: when
it runs out the kernel sets ``LH_STATUS_TIMEOUT`` in its status word, finishes
its own copies, frees its tensor memory and returns, and the host raises
instead of hanging. ``lh_wait_selftest`` makes one such wait run out (an
mbarrier that nothing completes, 20 ms limit); the context must stay usable:
the fused flash kernel then matches the reference's outputs as before.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT_NS = 20_000_000


def test_bounded_wait_reports_and_the_context_stays_usable(flash_table, flash_config,
                                                           flash_golden):
    import torch
    from lighthit_b200 import _lib
    from lighthit_b200.flash import FlashTransport
    from lighthit_b200.model import synthetic_detector
    lib = _lib.load()
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    stream = _lib.stream_ptr(torch.cuda.current_stream())
    _lib.check(lib.lh_wait_selftest(status.data_ptr(), LIMIT_NS, stream), "lh_wait_selftest")
    torch.cuda.synchronize()
    host = status.cpu().numpy()
    assert host[0] & _lib.LH_STATUS_TIMEOUT
    waited = int(host[2:4].view(np.uint64)[0])
    assert LIMIT_NS <= waited < 50 * LIMIT_NS, waited
    # invalid limits are refused before any launch
    assert lib.lh_wait_selftest(status.data_ptr(), 0, stream) == _lib.LH_EINVAL
    assert lib.lh_wait_selftest(status.data_ptr(), 2_000_000_000, stream) == _lib.LH_EINVAL
    # the context is intact: the fused tcgen05 flash kernel runs and matches
    g = flash_golden
    ft = FlashTransport(synthetic_detector(), flash_config, flash_table, mode="split-bf16")
    out = ft.run(g["flash_position_m"], g["flash_photons"], g["flash_time_ns"])
    charge = out["charge"].cpu().numpy().sum(axis=2)
    ref = g["charge_components_pe"].sum(axis=2)
    big = ref >= float(g["threshold_pe"])
    assert np.all(np.abs(charge[big] - ref[big]) <= 1e-3 * np.abs(ref[big]))
    assert not np.any(out["active"].cpu().numpy() & 6)
