"""The C-ABI library loads and exports every symbol the header declares (no GPU calls)."""
import ctypes
import re

from conftest import ROOT


def declared_symbols():
    text = (ROOT / "include" / "lighthit_b200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char\s*\*)\s+(lh_\w+)\s*\(", text,
                                 flags=re.M)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "lh_flash_transport" in names and "lh_readout_rows" in names


def test_library_exports_every_declared_symbol():
    from lighthit_b200 import _lib
    from lighthit_b200.build import build
    build()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert set(declared_symbols()) == set(_lib.SIGNATURES)
    loaded = _lib.load()
    assert loaded.lh_version().decode().startswith("lighthit_b200")
