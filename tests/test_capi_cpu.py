"""The C-ABI library without a GPU: it loads, exports every declared entry
point, and rejects invalid arguments before touching the device."""

import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "redi_b200.h")


def _declared():
    src = open(HEADER).read()
    return re.findall(r"^REDI_B200_API\s+[\w\s\*]*?\b(\w+)\s*\(", src, flags=re.M)


def test_header_declares_entry_points():
    names = _declared()
    for n in ("redi_b200_init", "redi_b200_calc_coeffs", "redi_b200_apply_flux", "redi_b200_destroy",
              "redi_opt_launch", "redi_cuda_launch_"):
        assert n in names


def test_every_declared_symbol_is_exported(redi_lib):
    L = redi_lib.lib()
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing


def test_version(redi_lib):
    assert redi_lib.lib().redi_b200_version() == 100


def test_init_rejects_bad_arguments_without_a_device(redi_lib):
    R = redi_lib
    L = R.lib()
    g = R.HGrid(20, 16, 16, 12, 2)._c()
    h = C.c_void_p(0)
    assert L.redi_b200_init(C.byref(g), 10, 0, None) == R.E_ARG
    assert L.redi_b200_init(None, 10, 0, C.byref(h)) == R.E_ARG
    assert L.redi_b200_init(C.byref(g), 10, 7, C.byref(h)) == R.E_ARG
    assert L.redi_b200_init(C.byref(g), 100000, 0, C.byref(h)) == R.E_UNSUPPORTED
    assert "exceeds" in R.last_error()
    bad = R.HGrid(0, 16, 16, 12, 2)._c()
    assert L.redi_b200_init(C.byref(bad), 10, 0, C.byref(h)) == R.E_ARG
    assert L.redi_b200_destroy(None) == R.OK


def test_calls_on_null_handles_are_errors(redi_lib):
    R = redi_lib
    L = R.lib()
    assert L.redi_b200_set_enable(None, 1) == R.E_ARG
    assert L.redi_b200_calc_coeffs(None, None, None, None, None, None) == R.E_ARG
    assert L.redi_b200_apply_flux(None, None, None, None, 1.0, None, None, None, None) == R.E_ARG


def test_compat_launcher_rejects_null_scalars(redi_lib, capfd):
    R = redi_lib
    L = R.lib()
    L.redi_opt_launch(*([None] * 42))
    assert "NULL scalar" in R.last_error()
    assert "redi_opt_launch" in capfd.readouterr().err


def test_product_path_has_no_cpu_fallback(redi_lib, tmp_path, monkeypatch):
    """Without the built library the host mirror raises instead of computing anything."""
    R = redi_lib
    monkeypatch.setattr(R, "_lib", None)
    monkeypatch.setattr(R, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(RuntimeError, match="missing"):
        R.lib()
