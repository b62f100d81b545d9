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


def test_omega_validation_and_short_range_rejected_without_gpu():
    # omega follows plan.py:18-27; env[8] < 0 (short range) is refused by the
    # table validation, before any device work
    import numpy as np
    from gradscf_b200 import _capi
    from gradscf_b200 import basis as B
    from gradscf_b200.jk import validate_omega
    assert validate_omega(0) == 0.0 and validate_omega(0.33) == 0.33
    for bad, exc in ((-0.1, ValueError), (float("nan"), ValueError), (True, TypeError), ("0.3", TypeError)):
        with pytest.raises(exc):
            validate_omega(bad)
    top, par, _ = B.prepare_basis("H 0 0 0; H 0 0 0.74", "sto-3g", cart=False)
    atm, bas, env = (np.ascontiguousarray(x) for x in B.pack(top, par))
    env = env.astype(np.float64).copy()
    env[8] = -0.3
    mol = _capi.Molecule(atm.ctypes.data, atm.shape[0], bas.ctypes.data, bas.shape[0],
                         env.ctypes.data, env.shape[0])
    arr = (_capi.Molecule * 1)(mol)
    h = ctypes.c_void_p()
    rc = _capi.lib().b200jk_plan_create(arr, 1, 0, 0.0, 0, ctypes.byref(h))
    assert rc == _capi.UNSUPPORTED and b"Short-range" in _capi.lib().b200jk_last_error()
