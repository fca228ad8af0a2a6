"""Device readout GEMM (fp32 CUDA cores, tcgen05 BF16 / split-BF16) vs the oracle."""
import numpy as np
import pytest

from conftest import GOLDEN
from oracle.readout import readout_bins

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode,tol", [("fp32", 1e-5), ("split-bf16", 5e-5), ("bf16", 2e-2)])
@pytest.mark.parametrize("rows", [1, 10, 127, 128, 129, 1000])
def test_readout_rows_match_oracle(mode, tol, rows):
    import torch
    from lighthit_b200.readout import DeviceReadout
    g = np.load(GOLDEN / "readout_c0.npz")
    ro = DeviceReadout(g["omega_per_ns"], g["edges_ns"], g["readout_omega_per_ns"])
    rng = np.random.default_rng(rows)
    rel = (rng.normal(size=(65, rows)) + 1j * rng.normal(size=(65, rows))) * np.exp(
        -np.linspace(0, 4, 65))[:, None]
    ref = readout_bins(g["omega_per_ns"], rel, g["edges_ns"], g["readout_omega_per_ns"])
    out, status = ro.bins(torch.tensor(rel.T.astype(np.complex64), device="cuda"), mode=mode)
    torch.cuda.synchronize()
    assert int(status[0]) == 0
    got = out.cpu().numpy()
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()


def test_readout_many_bin_tiles():
    """2060 bins (1 ns from -60 to 2000 ns) on a 1025-node readout grid: 9 N tiles."""
    import torch
    from lighthit_b200.readout import DeviceReadout
    omega = np.linspace(0, 1.2, 65)
    edges = np.arange(-60.0, 2001.0, 1.0)
    readout = np.linspace(0, 1.2, 1025)
    ro = DeviceReadout(omega, edges, readout)
    assert ro.n_tiles > 1
    rng = np.random.default_rng(3)
    rel = (rng.normal(size=(65, 300)) + 1j * rng.normal(size=(65, 300))) * np.exp(
        -np.linspace(0, 4, 65))[:, None]
    ref = readout_bins(omega, rel, edges, readout)
    for mode, tol in (("fp32", 1e-5), ("split-bf16", 5e-5)):
        out, status = ro.bins(torch.tensor(rel.T.astype(np.complex64), device="cuda"), mode=mode)
        torch.cuda.synchronize()
        assert int(status[0]) == 0
        assert np.abs(out.cpu().numpy() - ref).max() <= tol * np.abs(ref).max()
