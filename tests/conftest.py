import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"
TABLES = ROOT / "lighthit_b200" / "tables"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def flash_golden():
    return np.load(GOLDEN / "flash_c1.npz")


@pytest.fixture(scope="session")
def flash_table():
    from lighthit_b200.flash import FlashTable
    return FlashTable.load(TABLES / "flash_450nm_2-250m.npz")


@pytest.fixture(scope="session")
def flash_config(flash_golden):
    from lighthit_b200.model import KernelConfig
    g = flash_golden
    return KernelConfig(omega_per_ns=g["omega_per_ns"], readout_omega_per_ns=g["readout_omega_per_ns"],
                        relative_time_edges_ns=g["edges_ns"], radial_range_m=(2.0, 250.0),
                        threshold_pe=float(g["threshold_pe"]))


def oracle_detector(golden):
    return dict(positions_m=golden["om_positions_m"], orientations=golden["om_orientations"],
                area_m2=golden["om_area_m2"], alpha=golden["alpha"],
                acceptance=lambda x: .45 + .45 * np.asarray(x) + .10 * np.asarray(x) ** 2,
                spectral_weight=float(golden["spectral_weight_450"]))


def oracle_config(golden):
    return dict(omega_per_ns=golden["omega_per_ns"], readout_omega_per_ns=golden["readout_omega_per_ns"],
                edges_ns=golden["edges_ns"], threshold_pe=float(golden["threshold_pe"]),
                radial_range_m=(2.0, 250.0))
