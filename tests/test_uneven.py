"""Batched uneven correlation in one CUDA graph (needs a B200): raster pairs of different sizes and
tile geometries, each geometry autotuned, all work replayed as one graph launch.  The replay must
reproduce the eager results bit for bit, and every pair of every job passes the pair-by-pair
oracle check (oracle.parity.compare: cells equal to the FP64 oracle's unless the pair's own
surface error explains a near-tie, offsets then bit-exact)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import parity
from ampcor_b200 import batch
from ampcor_b200.worker import DIAG_DTYPE


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
        w = ub.workers[j.geometry]
        P = j.pairs
        dev = j.ref.device
        diag = torch.zeros((P, DIAG_DTYPE.itemsize), dtype=torch.uint8, device=dev)
        cs = torch.zeros((P, w.coarse_dim, w.coarse_dim), dtype=torch.float32, device=dev)
        rs = torch.zeros((P, w.refined_dim, w.refined_dim), dtype=torch.float32, device=dev)
        off = w.correlate(j.ref, j.tgt, ub.ulhc[k], diag=diag, coarse_surfaces=cs,
                          refined_surfaces=rs)
        assert np.array_equal(off.cpu().numpy(), eager[k]), k
        W = j.chip + 2 * j.margin
        orc = parity.oracle_run(j.ref.cpu().numpy(), j.tgt.cpu().numpy(), j.ulhc, j.chip, W,
                                j.refine_factor, j.refine_margin, j.zoom_factor)
        rep = parity.compare(orc, eager[k], diag.cpu().numpy().view(DIAG_DTYPE).reshape(P),
                             cs.cpu().numpy(), rs.cpu().numpy())
        assert not rep["failures"], (k, parity.summary(rep))
        assert rep["pairs_excused"] <= max(2, P // 100), (k, parity.summary(rep))
    ub.close()
