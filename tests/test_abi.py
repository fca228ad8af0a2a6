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


def test_ctypes_structs_match_the_c_layout(tmp_path):
    """Every ctypes struct has the size and field offsets gcc gives the header's struct."""
    import shutil
    import subprocess
    from lighthit_b200 import _lib
    pairs = {"lh_readout_operator": _lib.ReadoutOperator, "lh_flash_problem": _lib.FlashProblem,
             "lh_flash_batch": _lib.FlashBatch, "lh_ge2_table": _lib.Ge2Table,
             "lh_ge2_problem": _lib.Ge2Problem, "lh_order0_optics": _lib.Order0Optics,
             "lh_order0_batch": _lib.Order0Batch, "lh_order1_config": _lib.Order1Config,
             "lh_order1_elements": _lib.Order1Elements,
             "lh_order1_pencil_table": _lib.Order1PencilTable,
             "lh_source_problem": _lib.SourceProblem, "lh_source_output": _lib.SourceOutput,
             "lh_om_geometry_problem": _lib.OmGeometry, "lh_window_event": _lib.WindowEvent,
             "lh_radial_window_problem": _lib.RadialWindowProblem,
             "lh_near_table": _lib.NearTable, "lh_near_problem": _lib.NearProblem,
             "lh_flash_nodes": _lib.FlashNodes}
    cc = shutil.which("gcc") or shutil.which("cc")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "lighthit_b200.h"',
             "int main(void) {"]
    for cname, cls in pairs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            name, field, value = line.split()
            got[(name, field)] = int(value)
    for cname, cls in pairs.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)
