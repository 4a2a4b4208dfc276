"""Failure detection without a GPU fault (needs a B200).

Every wait of the tensor-core kernels and of the staged spectral correlation kernels (one
resident CTA per SM, windows brought in by the copy engine) is bounded in time; an expired wait
sets an error flag, the kernel stops issuing work, lets the work it issued finish, frees its
tensor memory and returns, and the host reports the time-out.  Here a wait is made to run out on
purpose, on a barrier that nothing completes (ampcor_inject_timeout), before any copy or
tensor-core work is issued: the batch must report AMPCOR_E_CUDA with the time-out message and the
same worker must then run the next batch to the same offsets as before.
"""
import numpy as np
import pytest

from ampcor_b200 import synth
from ampcor_b200.worker import Error, Worker

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _device(w):
    dev = torch.device("cuda:0")
    return (torch.from_numpy(w.ref).to(dev), torch.from_numpy(w.tgt).to(dev),
            torch.from_numpy(w.ulhc).to(dev))


@pytest.mark.parametrize("form", ["spectral", "tensor"])
def test_expired_wait_is_reported_and_the_worker_recovers(form):
    w = synth.plain_512()
    worker = Worker(pairs=w.pairs, chip=(32, 32), window=(48, 48), refine_factor=2,
                    refine_margin=4, zoom_factor=4)
    worker.configure(form)
    ref, tgt, u = _device(w)
    want = worker.correlate(ref, tgt, u).cpu().numpy().copy()
    worker.inject_timeout(1)
    with pytest.raises(Error) as e:
        worker.correlate(ref, tgt, u)
    assert "AMPCOR_E_CUDA" in str(e.value) and "timed out" in str(e.value)
    again = worker.correlate(ref, tgt, u).cpu().numpy()
    assert np.array_equal(again, want)
    worker.close()


def test_plain_form_has_no_bounded_waits_to_expire():
    w = synth.plain_512()
    worker = Worker(pairs=w.pairs, chip=(32, 32), window=(48, 48), refine_factor=2,
                    refine_margin=4, zoom_factor=4, plain=True)
    with pytest.raises(Error) as e:
        worker.inject_timeout(1)
    assert "AMPCOR_E_STATE" in str(e.value)
    worker.close()
