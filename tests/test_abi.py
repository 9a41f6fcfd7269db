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


# entry points that take a context first; called with a null context (and
# null or zero for everything else) each returns SNAP_ERR_BAD_ARG with a
# message, before touching a device
NULL_CTX_EXEMPT = {
    "snap_create", "snap_destroy", "snap_scratch_bytes", "snap_sweep_noalloc",
    "snap_selftest_division", "snap_last_error",
}


@pytest.mark.skipif(not LIB.exists(), reason="library not built")
def test_null_context_is_rejected():
    import sys
    sys.path.insert(0, str(ROOT / "legion-snap_b200"))
    from snap_b200 import abi
    lib = abi.load()
    for name, argtypes in abi.SIGNATURES.items():
        if name in NULL_CTX_EXEMPT:
            continue
        args = [0.0 if t is ctypes.c_double else 0 if t in (ctypes.c_int, ctypes.c_longlong)
                else None for t in argtypes]
        rc = getattr(lib, name)(*args)
        assert abi.STATUS.get(rc) == "SNAP_ERR_BAD_ARG", (name, rc)
        assert lib.snap_last_error(), name


@pytest.mark.skipif(not LIB.exists(), reason="library not built")
def test_create_rejects_null_arguments():
    import sys
    sys.path.insert(0, str(ROOT / "legion-snap_b200"))
    from snap_b200 import abi
    lib = abi.load()
    h = ctypes.c_void_p()
    assert abi.STATUS.get(lib.snap_create(None, 0, ctypes.byref(h))) == "SNAP_ERR_BAD_ARG"
    assert abi.STATUS.get(lib.snap_create(None, 0, None)) == "SNAP_ERR_BAD_ARG"
    assert lib.snap_destroy(None) in (0, 1)   # destroying nothing is harmless


def test_profiling_cases_cli(monkeypatch):
    """The single-kernel profiling cases the profile summaries name parse
    their documented command lines (no GPU call: parsing only)."""
    monkeypatch.syspath_prepend(str(ROOT / "legion-snap_b200"))
    from snap_b200 import cases
    called = {}
    for name in ("sweep_case", "outer_source_case", "input_deck_case", "adjoint_case"):
        monkeypatch.setattr(cases, name, lambda *a, _n=name: called.setdefault(_n, a))
    cases.main(["sweep", "--deck", "2", "--groups", "4", "--precision", "fp32"])
    cases.main(["outer-source", "--deck", "2", "--form", "tcgen05", "--calls", "3"])
    cases.main(["input-deck", "tests/decks/tiny_4K_1x1x1.in", "--inners", "3"])
    cases.main(["adjoint", "--deck", "4"])
    assert called["sweep_case"] == (2, 4, "fp32", 3)
    assert called["outer_source_case"] == (2, "tcgen05", 3)
    assert called["input_deck_case"] == ("tests/decks/tiny_4K_1x1x1.in", 3, False)
    assert called["adjoint_case"] == (4,)
