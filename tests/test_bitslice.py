"""The bitsliced AES-128 (cuot_b200/csrc/aes_bitslice.cuh, generated S-box
circuit bitslice_sbox.cuh): the S-box generator's own check, the core run on
the host against the oracle's FIPS-197 AES, and (GPU) the kernel against the
oracle and the T-table kernel."""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

import oracle
from tests.util import rng_blocks, to_dev, to_host

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cuot_b200", "csrc")


def test_sbox_generator_verifies_and_matches_committed_header(tmp_path):
    gen = os.path.join(CSRC, "gen_bitslice_sbox.py")
    work = tmp_path / "csrc"
    work.mkdir()
    shutil.copy(gen, work / "gen_bitslice_sbox.py")
    out = subprocess.run([sys.executable, str(work / "gen_bitslice_sbox.py")], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert "verified on all 256 inputs" in out.stdout
    assert (work / "bitslice_sbox.cuh").read_text() == open(os.path.join(CSRC, "bitslice_sbox.cuh")).read()


def test_bitsliced_core_on_host_matches_fips_aes(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("no nvcc")
    oracle.lib()  # builds liboracle.so if needed
    exe = str(tmp_path / "test_bitslice_host")
    subprocess.check_call([nvcc, "-std=c++17", "-O1", "-I", CSRC, "-I", os.path.join(ROOT, "include"),
                           "-I", os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "cpp", "test_bitslice_host.cu"),
                           os.path.join(ROOT, "oracle", "liboracle.so"), f"-Xlinker=-rpath={os.path.join(ROOT, 'oracle')}",
                           "-o", exe])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 31, 1024, 1025, 100003, 1 << 20])
def test_bitsliced_kernel_matches_oracle_and_ttable(ctx, n):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(n)
    key, pt = rng_blocks(rng, 1)[0], rng_blocks(rng, n)
    a, b = to_dev(pt), to_dev(pt)
    ctx.aes128_ecb_bitsliced(key, a)
    ctx.aes128_ecb(key, b)
    torch.cuda.synchronize()
    got = to_host(a)
    assert np.array_equal(got, to_host(b))
    if n <= 100003:
        assert np.array_equal(got, oracle.aes_ecb(key, pt))
