"""The C-ABI library loads and exports every declared symbol (no GPU calls)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "b200jk.h").read_text()
    return sorted(set(re.findall(r"\b(b200jk_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from gradscf_b200 import _capi
    if not _capi.LIB_PATH.exists():
        pytest.fail("libb200jk.so is not built; run python -m gradscf_b200.build")
    h = ctypes.CDLL(str(_capi.LIB_PATH))
    names = declared_symbols()
    assert "b200jk_direct_jk" in names and "b200jk_plan_create" in names
    for name in names:
        assert hasattr(h, name), name
    assert set(_capi.EXPORTS) <= set(names)


def test_last_error_is_callable_without_gpu():
    from gradscf_b200 import _capi
    assert _capi.lib().b200jk_last_error() is not None
