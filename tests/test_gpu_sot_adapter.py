"""The SOT role adapter (include/cuot_sot.h: SOTSender / SOTRecver with the
reference's interface), driven by a C++ program as a caller of cuOT's silent/
classes would, checked against the oracle and the COT correlation."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_test_binary(out_dir: str) -> str:
    exe = os.path.join(out_dir, "test_sot")
    cuda = "/usr/local/cuda"
    cmd = ["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "test_sot.cpp"),
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "oracle"), "-I", f"{cuda}/include",
           os.path.join(ROOT, "cuot_b200", "libcuot.so"), os.path.join(ROOT, "oracle", "liboracle.so"),
           f"-L{cuda}/lib64", "-lcudart", "-lpthread",
           f"-Wl,-rpath,{os.path.join(ROOT, 'cuot_b200')}:{os.path.join(ROOT, 'oracle')}:{cuda}/lib64",
           "-o", exe]
    subprocess.check_call(cmd)
    return exe


def test_sot_adapter_builds(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    assert os.path.exists(build_test_binary(str(tmp_path)))


@pytest.mark.gpu
def test_sot_adapter_matches_oracle(tmp_path):
    exe = build_test_binary(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr
