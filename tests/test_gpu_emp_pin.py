"""GPU tests: the CUDA path against the reference's OWN emp-ot code.

oracle/_ref/libempref.so holds ferret/emp-ot/emp-ot/ferret/{twokeyprp,
spcot_sender,spcot_recver,lpn_f2}.h compiled from the reference tree (over
the emp-tool shim in oracle/emp_shim), and oracle/_ref/test_emp_callers is
emp-ot's own MpcotReg / OTPre / LpnF2 callers compiled against
include/cuot_dev_layer.h and linked to libcuot.so.  Both are built where the
reference tree exists (oracle/build_ref.sh) and travel with the repository.
Every comparison is bit-exact.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
from tests.util import rng_blocks, delta_ferret, to_dev, to_host

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CALLERS = os.path.join(ROOT, "oracle", "_ref", "test_emp_callers")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(oracle.emp_lib() is None,
                                 reason="oracle/_ref/libempref.so not built (needs the reference tree)")]
torch = pytest.importorskip("torch")


def empty_blocks(n):
    return torch.empty((n, 16), dtype=torch.uint8, device="cuda")


def gpu_ferret(ctx, roots, h, delta, choice):
    t = roots.shape[0]
    lv, ls, rs, ss = empty_blocks(t << h), empty_blocks(t * h), empty_blocks(t * h), empty_blocks(t)
    ctx.ferret_pprf_sender(to_dev(roots), h, delta, lv, ls, rs, ss)
    mc = torch.where(to_dev(choice)[:, None] == 0, ls, rs)
    rl = empty_blocks(t << h)
    ctx.ferret_pprf_recver(mc, to_dev(choice), ss, h, rl)
    return lv, ls, rs, ss, rl


def test_c1_pprf_and_lpn_equal_reference_code(ctx):
    """The reference's CPU-runnable configuration (t = 64 trees of depth 10,
    k = 8,192, d = 10): the GPU sender's leaves, OT messages and secret sums
    equal SPCOT_Sender::compute, the receiver's leaves SPCOT_Recver::compute,
    and both roles' LPN outputs LpnF2::task over [0, n)."""
    rng = np.random.default_rng(2101)
    t, h, k = 64, 10, 8192
    roots, delta = rng_blocks(rng, t), delta_ferret(rng)
    choice = rng.integers(0, 2, t * h).astype(np.uint8)
    lv, ls, rs, ss, rl = gpu_ferret(ctx, roots, h, delta, choice)
    rlv, rm0, rm1, rss = oracle.emp_spcot_sender(roots, h, delta)
    assert np.array_equal(to_host(lv), rlv)
    assert np.array_equal(to_host(ls), rm0) and np.array_equal(to_host(rs), rm1)
    assert np.array_equal(to_host(ss), rss)
    mc = np.where(choice[:, None] == 0, rm0, rm1)
    rrl, _ = oracle.emp_spcot_recver(mc, choice, rss, h)
    assert np.array_equal(to_host(rl), rrl)
    seed, kk_s, kk_r = rng_blocks(rng, 1)[0], rng_blocks(rng, k), rng_blocks(rng, k)
    ctx.lpn_primal(seed, to_dev(kk_s), lv)
    ctx.lpn_primal(seed, to_dev(kk_r), rl)
    assert np.array_equal(to_host(lv), oracle.emp_lpn_task(seed, kk_s, rlv))
    assert np.array_equal(to_host(rl), oracle.emp_lpn_task(seed, kk_r, rrl))


def test_ferret_b13_sample_equals_reference_code(ctx):
    """ferret_b13 at full size on the GPU (t = 1,280 trees of depth 13,
    n = 10,485,760, k = 452,000): a seeded sample of 24 trees against
    SPCOT_Sender / SPCOT_Recver, and LPN rows against LpnF2::task on row
    windows.  A task over [s, e + 4) computes rows [s, e) in groups of four
    exactly as the single task over [0, n) does (its own __compute1 tail falls
    on rows e..e+3), and the last window ends at n, where the single task's
    tail lies."""
    rng = np.random.default_rng(1313)
    t, h, k = 1280, 13, 452000
    n = t << h
    roots, delta = rng_blocks(rng, t), delta_ferret(rng)
    choice = rng.integers(0, 2, t * h).astype(np.uint8)
    lv, ls, rs, ss, rl = gpu_ferret(ctx, roots, h, delta, choice)
    hl, hls, hrs, hss, hrl = (to_host(x) for x in (lv, ls, rs, ss, rl))
    for i in sorted(rng.choice(t, 24, replace=False).tolist()) + [0, t - 1]:
        rlv, rm0, rm1, rss = oracle.emp_spcot_sender(roots[i:i + 1], h, delta)
        assert np.array_equal(hl[i << h:(i + 1) << h], rlv), i
        assert np.array_equal(hls[i * h:(i + 1) * h], rm0) and np.array_equal(hrs[i * h:(i + 1) * h], rm1), i
        assert np.array_equal(hss[i], rss[0]), i
        mc = np.where(choice[i * h:(i + 1) * h, None] == 0, rm0, rm1)
        rrl, _ = oracle.emp_spcot_recver(mc, choice[i * h:(i + 1) * h], rss, h)
        assert np.array_equal(hrl[i << h:(i + 1) << h], rrl), i
    seed, kk = rng_blocks(rng, 1)[0], rng_blocks(rng, k)
    ctx.lpn_primal(seed, to_dev(kk), lv)
    got = to_host(lv)
    exp = hl.copy()
    # disjoint windows (each task also rewrites its 4 tail rows, never compared)
    starts = [((i * n) // 10 + int(rng.integers(0, 100000))) // 4 * 4 for i in range(1, 9)]
    windows = [(0, 4096)] + [(s, s + 4096) for s in starts]
    for s, e in windows:
        oracle.emp_lpn_task(seed, kk, exp, start=s, end=e + 4, inplace=True)
        assert np.array_equal(got[s:e], exp[s:e]), (s, e)
    oracle.emp_lpn_task(seed, kk, exp, start=n - 4096, end=n, inplace=True)
    assert np.array_equal(got[n - 4096:], exp[n - 4096:])


@pytest.mark.parametrize("n", [1, 3, 4, 5, 6, 7, 8, 9, 63, 64, 65, 66, 67, 4099])
def test_lpn_tails_equal_reference_code(ctx, n):
    """n mod 4 in {0, 1, 2, 3} and n <= 4: LpnF2::task's __compute1 tail."""
    rng = np.random.default_rng(4000 + n)
    k = 100 + 7 * n
    kk, e, seed = rng_blocks(rng, k), rng_blocks(rng, n), rng_blocks(rng, 1)[0]
    d = to_dev(e)
    ctx.lpn_primal(seed, to_dev(kk), d)
    assert np.array_equal(to_host(d), oracle.emp_lpn_task(seed, kk, e))


def test_emp_callers_through_the_adapter():
    """emp-ot's MpcotReg::exec_parallel_sender/recver (with OTPre carrying
    the level sums) and LpnF2::compute, compiled against
    include/cuot_dev_layer.h, run on libcuot.so and agree with
    SPCOT_Sender/SPCOT_Recver::compute and LpnF2::task; cases t = 64, h = 10,
    k = 8,192; t = 37, h = 9, k = 3,001; t = 20, h = 13, k = 452,000."""
    if not os.path.exists(CALLERS):
        pytest.skip("oracle/_ref/test_emp_callers not built (needs the reference tree)")
    r = subprocess.run([CALLERS], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr


@pytest.mark.parametrize("n,k,d", [(65536, 8192, 10), (4099, 1000, 10), (7, 33, 10), (1, 5, 10),
                                   (1030, 777, 7), (64, 200, 3)])
def test_dual_role_lpn_equals_reference_code_per_role(ctx, n, k, d):
    """cuot_lpn_primal_dual (both roles from one index computation) gives each
    role exactly LpnF2::task over [0, n) with that role's kk."""
    rng = np.random.default_rng(n + 13 * k + d)
    seed = rng_blocks(rng, 1)[0]
    kk_s, kk_r, e_s, e_r = rng_blocks(rng, k), rng_blocks(rng, k), rng_blocks(rng, n), rng_blocks(rng, n)
    ds, dr = to_dev(e_s), to_dev(e_r)
    ctx.lpn_primal_dual(seed, to_dev(kk_s), to_dev(kk_r), ds, dr, d=d)
    assert np.array_equal(to_host(ds), oracle.emp_lpn_task(seed, kk_s, e_s, d=d))
    assert np.array_equal(to_host(dr), oracle.emp_lpn_task(seed, kk_r, e_r, d=d))


def test_dual_role_lpn_full_size_b13(ctx):
    """ferret_b13 (n = 10,485,760, k = 452,000): the dual-role launch equals
    two single-role launches, bit for bit, on both roles."""
    rng = np.random.default_rng(1300)
    n, k = 10485760, 452000
    seed = rng_blocks(rng, 1)[0]
    kk_s, kk_r = to_dev(rng_blocks(rng, k)), to_dev(rng_blocks(rng, k))
    e_s = torch.randint(0, 256, (n, 16), dtype=torch.uint8, device="cuda")
    e_r = torch.randint(0, 256, (n, 16), dtype=torch.uint8, device="cuda")
    a_s, a_r = e_s.clone(), e_r.clone()
    ctx.lpn_primal_dual(seed, kk_s, kk_r, e_s, e_r)
    ctx.lpn_primal(seed, kk_s, a_s)
    ctx.lpn_primal(seed, kk_r, a_r)
    torch.cuda.synchronize()
    assert torch.equal(e_s, a_s) and torch.equal(e_r, a_r)
