"""CPU tests of the C ABI boundary: the library loads, exports every symbol
include/*.h declares, and its host-side argument checks behave without a GPU
(no compute is launched)."""
import ctypes
import os
import re

import pytest

import cuot_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    syms = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if not f.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", f)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        txt = re.sub(r"//[^\n]*", "", txt)
        # only the extern "C" entry points (C++ adapter headers are checked separately)
        if 'extern "C"' not in txt:
            continue
        syms |= set(re.findall(r"\b(cuot_[a-z0-9_]+)\s*\(", txt))
    return sorted(syms)


def test_library_exports_every_declared_symbol():
    lib = cuot_b200.load()
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert len(header_symbols()) >= 20


def test_version_and_status_strings():
    lib = cuot_b200.load()
    assert b"sm_100a" in lib.cuot_version()
    assert lib.cuot_status_string(0) == b"ok"
    assert lib.cuot_status_string(1) == b"invalid argument"
    assert lib.cuot_status_string(4) == b"timed out"


def test_ctx_create_rejects_bad_device():
    lib = cuot_b200.load()
    h = ctypes.c_void_p()
    st = lib.cuot_ctx_create(ctypes.c_int(-1), ctypes.byref(h))
    assert st == 1 and not h.value
    assert b"device" in lib.cuot_last_error()


def test_null_arguments_are_rejected_without_a_device():
    lib = cuot_b200.load()
    assert lib.cuot_ferret_pprf_sender(None, None, ctypes.c_uint64(1), 3, None, None, None, None, None, None) == 1
    assert lib.cuot_lpn_primal(None, None, None, ctypes.c_int64(1), 10, None, ctypes.c_int64(1), None) == 1
    assert lib.cuot_ctx_destroy(None) == 0
    assert lib.cuot_batch_wait_item(None, 0, None) == 1
    assert lib.cuot_batch_item_rank(None, 0) == -1


def test_server_arguments_are_checked_without_a_device():
    lib = cuot_b200.load()
    from cuot_b200.serve import _Config
    h = ctypes.c_void_p()
    assert lib.cuot_server_create(0, None, ctypes.byref(h)) == 1
    bad = _Config(slots=2, max_log_n=30, dry_run_service_s=0.01)
    assert lib.cuot_server_create(0, ctypes.byref(bad), ctypes.byref(h)) == 1
    assert b"max_log_n" in lib.cuot_last_error()
    assert lib.cuot_server_run(None, None, 0, None) == 1
    assert lib.cuot_server_destroy(None) == 0
