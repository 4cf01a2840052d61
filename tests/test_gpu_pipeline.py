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
