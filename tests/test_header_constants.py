"""The Python binding mirrors integer constants of include/cuot.h (tuning
keys, instance kinds, request states); the values must agree with the
header's #defines.  Reads the header as text (no device needed)."""
import os
import re

from cuot_b200 import Context
from cuot_b200 import batch, serve

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "cuot.h")


def defines() -> dict:
    out = {}
    for m in re.finditer(r"^#define\s+(CUOT_[A-Z0-9_]+)\s+(\d+)\b", open(HEADER).read(), re.M):
        out[m.group(1)] = int(m.group(2))
    return out


def test_tuning_keys():
    d = defines()
    for name in ("PPRF_THREADS", "QC_PLANES", "QC_BACKEND", "QC_STREAMS", "QC_RECORD_MARGIN"):
        assert getattr(Context, "TUNE_" + name) == d["CUOT_TUNE_" + name], name


def test_instance_kinds():
    d = defines()
    for mod in (batch, serve):
        assert mod.KIND_FERRET == d["CUOT_KIND_FERRET"] and mod.KIND_SOT == d["CUOT_KIND_SOT"]


def test_request_states():
    d = defines()
    for i, s in enumerate(serve.STATUS):
        assert d["CUOT_REQ_" + s.upper()] == i, s


def test_batch_schedules():
    d = defines()
    assert batch.FORK_FERRET == d["CUOT_BATCH_FORK_FERRET"]
    assert batch.SERIAL == d["CUOT_BATCH_SERIAL"]
    assert batch.FORK_SIZES == d["CUOT_BATCH_FORK_SIZES"]
