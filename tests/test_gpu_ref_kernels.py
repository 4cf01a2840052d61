"""GPU tests against the reference's own GPU kernels, rebuilt for sm_100a
from the reference tree (oracle/_ref/librefgpu.so, oracle/ref_gpu_driver.cu).

Of the reference's GPU outputs only Mat::bit_transpose is exact
(gpu/gpu_matrix.cu:95-121, bit_transposer gpu/gpu_ops.cu:31-70, for row
counts that are multiples of 256 up to 2^23); it pins this library's
transpose bit order against reference code run on the same GPU.  The timing
entry points (speed context for bench.py) are smoke-tested here.
"""
import numpy as np
import pytest

import oracle
from tests.util import rng_blocks, to_dev, to_host

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(oracle.refgpu_lib() is None,
                                 reason="oracle/_ref/librefgpu.so not built (needs the reference tree)")]
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("n", [256, 4096 + 256, 1 << 20, (1 << 23)])
def test_reference_bit_transposer_equals_ours(ctx, n):
    rng = np.random.default_rng(n)
    x = rng_blocks(rng, n)
    ref = oracle.refgpu_bit_transpose(x)
    out = torch.empty((128, n // 8), dtype=torch.uint8, device="cuda")
    ctx.bit_transpose(to_dev(x), n, 16, 0, 128, out)
    assert np.array_equal(to_host(out), ref)
    if n <= 4096 + 256:
        assert np.array_equal(oracle.bit_transpose(x, n, 16, 0, 128).reshape(128, n // 8), ref)


def test_reference_timing_entry_points_run():
    L = oracle.refgpu_lib()
    assert L.ref_gpu_mpcot_sender_ms(64, 10, 2) > 0
    assert L.ref_gpu_primal_lpn_ms(65536, 8192, 2) > 0
    assert L.ref_gpu_sot_dual_lpn_ms(1 << 17, 1) > 0
    # shapes outside the reference kernels' safe range are refused, not run
    assert L.ref_gpu_mpcot_sender_ms(1, 5, 1) < 0
    assert L.ref_gpu_primal_lpn_ms(1000, 10, 1) < 0
    assert L.ref_gpu_sot_dual_lpn_ms(1 << 16, 1) < 0
    assert L.ref_gpu_bit_transpose(None, 100, None) != 0
