"""HostPipeline (cuot_b200/pipeline.py): each step's results reach its own
host buffers intact although the host copy of step i overlaps step i+1,
which overwrites the device outputs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_pipeline_keeps_every_steps_results(ctx):
    from cuot_b200.pipeline import HostPipeline
    n = 1 << 22
    out = torch.empty((n, 16), dtype=torch.uint8, device="cuda")
    seed_d = torch.empty((1, 16), dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    pipe = HostPipeline([out], stream=st)
    hosts = [torch.empty((n, 16), dtype=torch.uint8).pin_memory() for _ in range(4)]
    seeds = [torch.full((1, 16), 11 * i + 1, dtype=torch.uint8).pin_memory() for i in range(4)]

    def compute(s, i):
        # device output = PRG stream of this step's seed (a long kernel), then the seed byte in row 0
        ctx.prg_fill(bytes([11 * i + 1] * 16), out, stream=s)
        with torch.cuda.stream(s):
            out[0].copy_(seed_d[0])
    for i in range(4):
        pipe.step([(seeds[i], seed_d)], lambda s, i=i: compute(s, i), [hosts[i]])
    pipe.join()
    st.synchronize()
    import oracle
    for i in range(4):
        h = hosts[i].numpy()
        assert (h[0] == 11 * i + 1).all()
        exp = oracle.prg(bytes([11 * i + 1] * 16), 1024)
        assert np.array_equal(h[1:1024], exp[1:1024])


def test_double_buffered_inputs_reach_their_own_step(ctx):
    """input_sets = 2: step j's input copy runs on its own stream while step
    j-1 computes; every step must still see its own inputs (a copy that
    overtook the last reader of its buffer set would show up as another
    step's seed)."""
    from cuot_b200.pipeline import HostPipeline
    n = 1 << 22
    out = torch.empty((n, 16), dtype=torch.uint8, device="cuda")
    seed_d = [torch.empty((1, 16), dtype=torch.uint8, device="cuda") for _ in range(2)]
    st = torch.cuda.Stream()
    pipe = HostPipeline([out], stream=st, input_sets=2)
    steps = 6
    hosts = [torch.empty((n, 16), dtype=torch.uint8).pin_memory() for _ in range(steps)]
    seeds = [torch.full((1, 16), 7 * i + 3, dtype=torch.uint8).pin_memory() for i in range(steps)]

    def compute(s, slot):
        # a long kernel first, so the next step's input copy has time to overtake
        ctx.prg_fill(bytes(16), out, stream=s)
        with torch.cuda.stream(s):
            out[0].copy_(seed_d[slot][0])
    for i in range(steps):
        slot = pipe.slot
        assert slot == i % 2
        pipe.step([(seeds[i], seed_d[slot])], lambda s, slot=slot: compute(s, slot), [hosts[i]])
    pipe.join()
    st.synchronize()
    for i in range(steps):
        assert (hosts[i].numpy()[0] == 7 * i + 3).all(), i


def test_copy_to_host_through_sm_stores(ctx):
    """cuot_copy_to_host: device bytes land in pinned host memory, with
    16-byte and byte-granular paths (aligned and odd sizes / offsets), two
    calls in a row; an unpinned destination is refused."""
    import cuot_b200
    rng = np.random.default_rng(3)
    for nbytes in (16 * 4097, 1000003):
        src = torch.from_numpy(rng.integers(0, 256, nbytes, dtype=np.uint8)).cuda()
        dst = torch.zeros(nbytes + 1, dtype=torch.uint8).pin_memory()
        for view in (dst[:nbytes], dst[1:]):
            view.zero_()
            cuot_b200.copy_to_host(src, view)
            torch.cuda.synchronize()
            assert np.array_equal(view.numpy(), src.cpu().numpy())
    import ctypes
    pageable = np.zeros(64, np.uint8)
    st = cuot_b200.load().cuot_copy_to_host(ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(pageable.ctypes.data),
                                            ctypes.c_uint64(64), None)
    assert st == 1 and b"mapped" in cuot_b200.load().cuot_last_error()
    with pytest.raises(ValueError):
        cuot_b200.copy_to_host(src[:16], torch.zeros(16, dtype=torch.uint8))
