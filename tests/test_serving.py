"""The continuous-batching request loop (needs a B200): every job's offsets are bitwise the same
whether it runs alone or overlapped with other jobs on the device, the offsets recover the
applied sub-pixel shifts, the served offsets pass the pair-by-pair oracle check on a sample of
every job over the full serving range (chips 32-128, margins 16-64, zoom 8-16), and a job larger
than the memory budget is refused while the others run."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import parity
from ampcor_b200 import serve
from ampcor_b200.worker import DIAG_DTYPE, Worker


def _jobs(pinned):
    return serve.poisson_jobs(10, rate=40.0, seed=7, sizes=(1024, 2048), chips=(32, 64),
                              margins=(16, 32), zooms=(8, 16), spacing=(96, 160), pinned=pinned)


@pytest.mark.parametrize("pinned", [False, True])
def test_same_alone_and_in_the_mix(pinned):
    jobs = _jobs(pinned)
    # alone: one slot, one job at a time
    alone = serve.Server(slots=1)
    alone.warm(jobs)
    for j in jobs:
        alone.run([j], realtime=False)
    ref = {j.jid: j.offsets.copy() for j in jobs}
    for j in jobs:
        j.offsets = j.done = j.start = None
    # in the mix: four slots, arrivals on the Poisson clock, kernels of different jobs overlap
    mixed = serve.Server(slots=4)
    mixed.warm(jobs)
    mixed.run(jobs, realtime=True)
    for j in jobs:
        assert np.array_equal(j.offsets, ref[j.jid]), j.jid
    rep = serve.latency_report(jobs)
    assert rep["jobs"] == len(jobs)
    # quantum 1/(2 z) px; the applied shifts are recovered to within it everywhere
    assert rep["max_offset_error_px"] < 0.1
    assert rep["p99_ms"] >= rep["p50_ms"] > 0


GEOMETRIES = [(32, 64, 16), (64, 16, 8), (128, 32, 8), (128, 64, 16), (64, 64, 8), (32, 16, 16)]


def _range_jobs():
    """One job per (chip, margin, zoom) across the serving range, on 1024-2048 px rasters."""
    jobs = []
    for k, (chip, margin, zoom) in enumerate(GEOMETRIES):
        lines, samples = (2048, 1024) if k % 2 else (1024, 2048)
        shift = (0.37 * k - 1.1, 2.3 - 0.61 * k)
        ref, tgt = serve.synth_pair(lines, samples, shift, 9001 + k, "cuda:0")
        ulhc = serve.grid_corners(lines, samples, chip, margin, 200)
        jobs.append(serve.Job(k, 0.01 * k, ref, tgt, ulhc, chip, margin, 2, 8, zoom, truth=shift))
    return jobs


def test_full_range_served_offsets_pass_the_oracle_check():
    # chips 32-128, margins 16-64, zoom 8-16 served together; a sample of each job's pairs rerun
    # alone with surfaces gives the served offsets bit for bit and passes oracle.parity.compare
    jobs = _range_jobs()
    srv = serve.Server(slots=3)
    srv.warm(jobs)
    srv.run(jobs, realtime=False)
    assert all(j.error is None for j in jobs)
    for j in jobs:
        sel = np.linspace(0, j.pairs - 1, min(12, j.pairs)).round().astype(int)
        ulhc = j.ulhc[sel]
        W = j.chip + 2 * j.margin
        w = Worker(pairs=len(sel), chip=(j.chip, j.chip), window=(W, W), refine_factor=j.refine_factor,
                   refine_margin=j.refine_margin, zoom_factor=j.zoom_factor)
        dev = j.ref.device
        P = len(sel)
        diag = torch.zeros((P, DIAG_DTYPE.itemsize), dtype=torch.uint8, device=dev)
        cs = torch.zeros((P, w.coarse_dim, w.coarse_dim), dtype=torch.float32, device=dev)
        rs = torch.zeros((P, w.refined_dim, w.refined_dim), dtype=torch.float32, device=dev)
        off = w.correlate(j.ref, j.tgt, torch.from_numpy(ulhc).to(dev), diag=diag,
                          coarse_surfaces=cs, refined_surfaces=rs).cpu().numpy()
        w.close()
        assert np.array_equal(off, j.offsets[sel]), j.jid
        orc = parity.oracle_run(j.ref.cpu().numpy(), j.tgt.cpu().numpy(), ulhc, j.chip, W,
                                j.refine_factor, j.refine_margin, j.zoom_factor)
        rep = parity.compare(orc, off, diag.cpu().numpy().view(DIAG_DTYPE).reshape(P),
                             cs.cpu().numpy(), rs.cpu().numpy())
        assert not rep["failures"], (j.jid, j.geometry, parity.summary(rep))
        assert np.abs(j.offsets - np.asarray(j.truth)[None, :]).max() < 0.1


def test_job_beyond_the_budget_is_refused_and_the_rest_run():
    jobs = serve.poisson_jobs(4, rate=40.0, seed=3, sizes=(1024,), chips=(32,), margins=(16,),
                              zooms=(8,), spacing=(128, 128), pinned=False)
    big = serve.poisson_jobs(1, rate=40.0, seed=5, sizes=(2048,), chips=(32,), margins=(16,),
                             zooms=(8,), spacing=(128, 128), pinned=False)[0]
    big.jid = 99
    jobs.insert(2, big)
    budget = max(j.device_bytes() for j in jobs if j is not big) * 2
    assert big.device_bytes() > budget
    srv = serve.Server(slots=2, memory_budget=budget)
    srv.warm([j for j in jobs if j is not big])
    srv.run(jobs, realtime=False)
    assert big.error and "budget" in big.error and big.offsets is None
    assert all(j.error is None and j.offsets is not None for j in jobs if j is not big)
    rep = serve.latency_report(jobs)
    assert rep["refused"] == 1 and rep["jobs"] == 4
