"""HostPipeline (cuot_b200/pipeline.py): every step's outputs reach the host
intact while the next steps compute, with staged outputs (one device set) and
with one device output set per input set (no staging copy; a set is written
again only after its previous results reached the host), and with per-output
completion points (`ready`)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from cuot_b200.pipeline import HostPipeline  # noqa: E402

N = 1 << 22  # int32 elements per output (16 MiB): each host copy takes a while


def _run(per_set: bool, steps: int = 6):
    st = torch.cuda.Stream()
    sets = 2 if per_set else 1
    outs = [[torch.empty(N, dtype=torch.int32, device="cuda") for _ in range(2)] for _ in range(sets)]
    ins = [torch.empty(4, dtype=torch.int32, device="cuda") for _ in range(2)]
    host_in = [torch.tensor([j, 0, 0, 0], dtype=torch.int32).pin_memory() for j in range(steps)]
    host_out = [[torch.empty(N, dtype=torch.int32).pin_memory() for _ in range(2)] for _ in range(steps)]
    pipe = HostPipeline(outs if per_set else outs[0], stream=st, input_sets=2, per_set_outputs=per_set)
    for j in range(steps):
        slot = pipe.slot
        o = outs[slot if per_set else 0]

        def compute(s, o=o, slot=slot):
            with torch.cuda.stream(s):
                torch.cuda._sleep(2_000_000)  # let the previous host copy still be running
                o[0].fill_(0).add_(ins[slot][0])  # the step's own input, copied in by the pipeline
                o[1].fill_(0).add_(ins[slot][0] * 3 + 1)
        h2d, d2h = pipe.step([(host_in[j], ins[slot])], compute, host_out[j])
        assert h2d == 16 and d2h == 2 * 4 * N
    pipe.join()
    torch.cuda.synchronize()
    for j in range(steps):
        assert (host_out[j][0].numpy() == j).all() and (host_out[j][1].numpy() == 3 * j + 1).all(), j


def test_pipeline_staged_outputs():
    _run(per_set=False)


def test_pipeline_per_set_outputs():
    _run(per_set=True)


def test_pipeline_per_set_outputs_need_one_list_per_set():
    t = torch.empty(4, device="cuda")
    with pytest.raises(ValueError):
        HostPipeline([[t]], input_sets=2, per_set_outputs=True)


def test_pipeline_per_output_ready_points():
    """With `ready`, each output's host copy waits only for its own
    completion point: output 0 is final early in the step, output 1 after a
    long sleep.  Both must reach the host intact (a missing wait would copy
    output 1 before the step wrote it)."""
    st = torch.cuda.Stream()
    steps = 4
    outs = [[torch.empty(N, dtype=torch.int32, device="cuda") for _ in range(2)] for _ in range(2)]
    ins = [torch.empty(4, dtype=torch.int32, device="cuda") for _ in range(2)]
    host_in = [torch.tensor([j, 0, 0, 0], dtype=torch.int32).pin_memory() for j in range(steps)]
    host_out = [[torch.empty(N, dtype=torch.int32).pin_memory() for _ in range(2)] for _ in range(steps)]
    pipe = HostPipeline(outs, stream=st, input_sets=2, per_set_outputs=True)
    for j in range(steps):
        slot = pipe.slot
        o = outs[slot]
        marks = [torch.cuda.Event(), torch.cuda.Event()]

        def compute(s, o=o, slot=slot, marks=marks):
            with torch.cuda.stream(s):
                o[0].fill_(0).add_(ins[slot][0])
                marks[0].record(s)
                torch.cuda._sleep(4_000_000)
                o[1].fill_(0).add_(ins[slot][0] * 5 + 2)
                marks[1].record(s)
        ready = [lambda cs, e=marks[0]: cs.wait_event(e), lambda cs, e=marks[1]: cs.wait_event(e)]
        pipe.step([(host_in[j], ins[slot])], compute, host_out[j], ready)
    pipe.join()
    torch.cuda.synchronize()
    for j in range(steps):
        assert (host_out[j][0].numpy() == j).all() and (host_out[j][1].numpy() == 5 * j + 2).all(), j


def test_pipeline_ready_is_checked():
    t = [torch.empty(4, device="cuda")]
    h = [torch.empty(4).pin_memory()]
    pipe = HostPipeline([t, t], input_sets=2, per_set_outputs=True)
    with pytest.raises(ValueError):
        pipe.step([], lambda s: None, h, [None])  # the first entry must wait
    with pytest.raises(ValueError):
        pipe.step([], lambda s: None, h, [])
    staged = HostPipeline(t)
    with pytest.raises(ValueError):
        staged.step([], lambda s: None, h, [lambda cs: None])
    torch.cuda.synchronize()
