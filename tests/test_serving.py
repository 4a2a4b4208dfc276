"""The continuous-batching request loop (needs a B200): every job's offsets are bitwise the same
whether it runs alone or overlapped with other jobs on the device, and the offsets recover the
applied sub-pixel shifts."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from ampcor_b200 import serve


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
