"""Batched uneven correlation in one CUDA graph (needs a B200): raster pairs of different sizes and
tile geometries, each geometry autotuned, all work replayed as one graph launch.  The replay must
reproduce the eager results bit for bit, and every job agrees with the FP64 oracle on a sample of
its pairs (integer offsets exact, sub-pixel cells equal away from near-ties)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import oracle
from ampcor_b200 import batch


def test_uneven_batch_graph_replay_and_parity():
    jobs = batch.uneven_jobs(n=5, seed=3, shapes=((1024, 1024), (2048, 1024), (1024, 1536)),
                             chips=(32, 64), margins=(8, 16, 32), spacing=(48, 96))
    ub = batch.UnevenBatch(jobs, tune=True)
    g = ub.capture()
    eager = [o.cpu().numpy().copy() for o in ub.offsets]
    for o in ub.offsets:
        o.fill_(float("nan"))
    ub.replay()
    torch.cuda.synchronize()
    ub.check()
    for k, (o, e) in enumerate(zip(ub.offsets, eager)):
        assert np.array_equal(o.cpu().numpy(), e), k
    for k, j in enumerate(jobs):
        n = min(12, j.pairs)
        sel = np.linspace(0, j.pairs - 1, n).round().astype(int)
        ref = j.ref.cpu().numpy()
        tgt = j.tgt.cpu().numpy()
        W = j.chip + 2 * j.margin
        want, od = oracle.adjust(ref, tgt, j.ulhc[sel], j.chip, W, j.refine_factor,
                                 j.refine_margin, j.zoom_factor)
        arg, gap = oracle.coarse_cpu(ref, tgt, j.ulhc[sel], j.chip, W)
        got = eager[k][sel]
        quantum = 1.0 / (j.refine_factor * j.zoom_factor)
        safe = (gap > 1e-5) & (od["zoom_gap"] > 1e-5)
        assert np.array_equal(got[safe], want[safe]), k
        assert np.abs(got - want).max() <= max(quantum, 1.0) + 1e-6
    ub.close()
