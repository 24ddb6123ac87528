"""The C-ABI library builds, loads without a GPU and exports what include/ declares."""
from __future__ import annotations

import ctypes
import re

import pytest

from conftest import ROOT


def declared_functions() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(sqb_[a-z0-9_]+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    from sqdft_b200.sq import EXPORTS

    assert set(EXPORTS) <= names, sorted(set(EXPORTS) - names)


def test_library_exports_every_declared_symbol():
    from sqdft_b200.build import build

    lib_path = build()
    lib = ctypes.CDLL(str(lib_path))
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_version_without_gpu():
    from sqdft_b200 import sq

    lib = sq.library()
    assert b"sm_100a" in lib.sqb_version()
    assert sq.status_string(0) == "ok"
    assert "bracketed" in sq.status_string(4)


def test_create_fails_cleanly_without_gpu(golden):
    """With no device the context constructor reports SQB_ERR_CUDA (no crash, no CPU path)."""
    from conftest import cuda_available
    from sqdft_b200 import sq

    if cuda_available():
        pytest.skip("a GPU is present")
    case, _ = golden("tiny")
    with pytest.raises(sq.SQBError) as ei:
        sq.Context(case)
    assert ei.value.code == 2


def test_create_rejects_bad_grid(golden):
    from sqdft_b200 import sq

    case, _ = golden("tiny")
    import dataclasses

    bad = dataclasses.replace(case, npl=30)  # npl must be a multiple of 4 (sq.cpp:523)
    with pytest.raises(sq.SQBError) as ei:
        sq.Context(bad)
    assert ei.value.code == 1
