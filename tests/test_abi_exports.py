"""CPU tests: the C-ABI library loads and exports every symbol the header declares."""

import re
from pathlib import Path

from sparkalog_b200 import _native

HEADER = Path(__file__).resolve().parent.parent / "include" / "sparkalog_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return re.findall(r"SPARKALOG_API\s+[\w\s\*]+?\b(sparkalog_\w+)\s*\(", text)


def test_header_declares_reference_operator_abi():
    names = set(declared_symbols())
    for name in ["sparkalog_stream_synchronize", "sparkalog_join_u32_temporary_bytes", "sparkalog_join_u32_count",
                 "sparkalog_join_u32_emit", "sparkalog_distinct_u32_temporary_bytes", "sparkalog_distinct_u32",
                 "sparkalog_anti_join_u32_temporary_bytes", "sparkalog_anti_join_u32",
                 "sparkalog_union_u32_temporary_bytes", "sparkalog_union_u32"]:
        assert name in names


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    declared = declared_symbols()
    assert declared
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) <= set(_native.EXPORTED) | set(declared)


def test_bindings_cover_the_header():
    assert set(_native.EXPORTED) == set(declared_symbols())


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    import pytest

    monkeypatch.setattr(_native, "LIB_PATH", tmp_path / "absent.so")
    monkeypatch.setattr(_native, "_lib", None)
    with pytest.raises(ImportError):
        _native.load()
