"""The C-ABI library loads and exports every entry point include/*.h
declares (no compute call: this runs without a GPU)."""
import ctypes
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
LIB = ROOT / "legion-snap_b200" / "snap_b200" / "libsnap_b200.so"


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names.update(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(snap_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("snap_create", "snap_sweep", "snap_calc_outer_source", "snap_calc_inner_source",
              "snap_expand_xs", "snap_test_convergence", "snap_transport_solve"):
        assert n in names


@pytest.mark.skipif(not LIB.exists(), reason="library not built")
def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(LIB))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.skipif(not LIB.exists(), reason="library not built")
def test_python_binding_covers_header():
    import sys
    sys.path.insert(0, str(ROOT / "legion-snap_b200"))
    from snap_b200 import abi
    assert set(declared_symbols()) <= set(abi.SIGNATURES)
