"""Autotuner: picks a configuration from measured candidates, persists it
keyed by shape, reuses it, and the tuned configuration gives the same
(bit-exact) outputs as the default one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from cuot_b200.autotune import TuningTable, batch_key, tune_batch, tune_single  # noqa: E402
from cuot_b200.batch import KIND_FERRET, KIND_SOT, Batch, Instance  # noqa: E402


def test_tune_batch_persists_and_preserves_outputs(ctx, tmp_path):
    insts = [Instance(ctx, KIND_SOT, 4, 10, 1), Instance(ctx, KIND_FERRET, 16, 10, 2, k=700),
             Instance(ctx, KIND_FERRET, 2, 13, 3, k=800)]
    table = TuningTable(str(tmp_path / "t.json"))
    cands = [dict(pprf_threads=128, ctas_per_sm=2, lpn_rows_per_task=4096),
             dict(pprf_threads=256, ctas_per_sm=3, lpn_rows_per_task=65536)]
    best, results = tune_batch(ctx, insts, table=table, candidates=cands)
    assert best in cands and len(results) == 2
    again = TuningTable(str(tmp_path / "t.json"))
    assert again.get(batch_key(insts))["config"] == best
    stream = torch.cuda.Stream()
    outs = []
    for cfg in cands:
        b = Batch(ctx, insts, **cfg)
        b.run(stream)
        torch.cuda.synchronize()
        outs.append([(i.v.cpu().numpy().copy(), i.w.cpu().numpy().copy()) for i in insts])
        b.close()
    for (v0, w0), (v1, w1) in zip(*outs):
        assert np.array_equal(v0, v1) and np.array_equal(w0, w1)


def test_tune_single_sets_context_knobs(ctx, tmp_path):
    inst = Instance(ctx, KIND_SOT, 8, 10, 5)
    hit = tune_single(ctx, inst, table=TuningTable(str(tmp_path / "s.json")))
    assert hit["pprf_threads"] in (128, 256) and hit["qc_planes_per_pass"] >= 1
    # restore the defaults for the other tests sharing this context
    ctx.set_tuning(ctx.TUNE_PPRF_THREADS, 256)
    ctx.set_tuning(ctx.TUNE_QC_PLANES, 0)
