"""CPU-side checks of the product library: it loads, exports every entry point declared in
include/b200fmm.h, and rejects bad arguments through status codes (no GPU needed for either)."""
import ctypes
import re
from pathlib import Path

import pytest

import scalfmm_b200 as S

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "b200fmm.h").read_text()
    return sorted(set(re.findall(r"B200FMM_API\s+[\w\s\*]*?\b(b200fmm_\w+)\s*\(", text)))


def test_header_and_binding_agree():
    assert sorted(S.EXPORTS) == declared_symbols()


def test_library_exports_every_declared_symbol():
    L = S.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name
    assert b"sm_100a" in L.b200fmm_version()


def test_invalid_configs_return_status_codes():
    L = S.lib()
    h = ctypes.c_void_p()
    bad = [
        S.Config(7, 5, 4, 1, 0, 1.0, (ctypes.c_double * 3)(0.5, 0.5, 0.5), 0.0, None, -1),   # kernel
        S.Config(0, 2, 4, 1, 0, 1.0, (ctypes.c_double * 3)(0.5, 0.5, 0.5), 0.0, None, -1),   # order
        S.Config(0, 5, 40, 1, 0, 1.0, (ctypes.c_double * 3)(0.5, 0.5, 0.5), 0.0, None, -1),  # height
        S.Config(0, 5, 4, 0, 0, 1.0, (ctypes.c_double * 3)(0.5, 0.5, 0.5), 0.0, None, -1),   # nrhs
        S.Config(0, 5, 4, 1, 9, 1.0, (ctypes.c_double * 3)(0.5, 0.5, 0.5), 0.0, None, -1),   # precision
        S.Config(0, 5, 4, 1, 0, -1.0, (ctypes.c_double * 3)(0.5, 0.5, 0.5), 0.0, None, -1),  # box
    ]
    for cfg in bad:
        assert L.b200fmm_create(ctypes.byref(cfg), ctypes.byref(h)) == 1  # B200FMM_ERR_INVALID
        assert h.value is None
    assert L.b200fmm_create(None, ctypes.byref(h)) == 1
    assert L.b200fmm_execute(None, 63) == 1
    assert L.b200fmm_destroy(None) == 0


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(S, "LIB_PATH", tmp_path / "nope.so")
    monkeypatch.setattr(S, "_lib", None)
    with pytest.raises(S.B200FmmError):
        S.lib()
