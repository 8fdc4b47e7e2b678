"""The C-ABI library loads and exports every symbol include/coral_b200.h
declares; the ctypes binding declares each of them.  No compute calls."""
import subprocess

from coral_b200 import _lib


def test_library_exports_header_symbols():
    lib = _lib.load()
    missing = [s for s in _lib.header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    assert sorted(_lib.SIGNATURES) == _lib.header_symbols()


def test_dynamic_symbol_table():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(_lib.header_symbols()) <= exported


def test_abi_version_and_status_strings():
    lib = _lib.load()
    assert lib.coral_abi_version() == 1
    assert lib.coral_status_string(0) == b"CORAL_OK"
    assert lib.coral_status_string(3) == b"CORAL_ERR_TIMEOUT"


def test_null_handle_is_rejected():
    lib = _lib.load()
    assert lib.coral_sync(None) == 1
    assert lib.coral_sgemm(None, 0, 0, 1, 1, 1, 1.0, None, 1, None, 1, 0.0, None, 1) == 1
