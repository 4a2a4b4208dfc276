"""The allocation-free entry point, ampcor_correlate_noalloc (needs a B200).

It exists for callers that cannot allocate device memory while they run (an application whose
own memory pool holds the whole GPU, or a real-time chain that forbids allocation after
start-up).  It must give the same offsets and diagnostics as the regular entry point,
ampcor_correlate, for the same batch, including on a second call right after the first (the
fixed scratch array keeps the previous call's contents).  This file is collected last so that a
run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from ampcor_b200 import _lib, synth
from ampcor_b200.worker import DIAG_DTYPE, Worker, torch_stream_handle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def params_of(w):
    return _lib.Params(pairs=0, ref_lines=w.chip, ref_samples=w.chip, tgt_lines=w.window,
                       tgt_samples=w.window, refine_factor=w.refine_factor,
                       refine_margin=w.refine_margin, zoom_factor=w.zoom_factor, device=0, flags=0)


def device_batch(w, ulhc):
    dev = torch.device("cuda:0")
    ref = torch.from_numpy(w.ref).to(dev)
    tgt = torch.from_numpy(w.tgt).to(dev)
    u = torch.from_numpy(np.ascontiguousarray(ulhc)).to(dev)
    return ref, tgt, u


def run_noalloc(w, ulhc):
    lib = _lib.load()
    ref, tgt, u = device_batch(w, ulhc)
    P = len(ulhc)
    off = torch.full((P, 2), float("nan"), dtype=torch.float32, device=ref.device)
    diag = torch.zeros((P, DIAG_DTYPE.itemsize), dtype=torch.uint8, device=ref.device)
    job = _lib.Job(ref=ref.data_ptr(), ref_lines=ref.shape[0], ref_samples=ref.shape[1],
                   tgt=tgt.data_ptr(), tgt_lines=tgt.shape[0], tgt_samples=tgt.shape[1],
                   ulhc=u.data_ptr(), pairs=P, offsets=off.data_ptr(), diag=diag.data_ptr())
    p = params_of(w)
    err = ctypes.create_string_buffer(256)
    st = ctypes.c_void_p(torch_stream_handle(None, ref.device))
    rc = lib.ampcor_correlate_noalloc(ctypes.byref(p), ctypes.byref(job), st, err, len(err))
    assert rc == _lib.OK, err.value.decode()
    return off.cpu().numpy(), diag.cpu().numpy().view(DIAG_DTYPE).reshape(P)


def run_regular(w, ulhc):
    # the allocation-free path runs the plain FP32 kernels: compare with the same form
    worker = Worker(pairs=len(ulhc), chip=(w.chip, w.chip), window=(w.window, w.window),
                    refine_factor=w.refine_factor, refine_margin=w.refine_margin,
                    zoom_factor=w.zoom_factor, plain=True)
    ref, tgt, u = device_batch(w, ulhc)
    diag = torch.zeros((len(ulhc), DIAG_DTYPE.itemsize), dtype=torch.uint8, device=ref.device)
    off = worker.correlate(ref, tgt, u, diag=diag)
    out = off.cpu().numpy(), diag.cpu().numpy().view(DIAG_DTYPE).reshape(len(ulhc))
    worker.close()
    return out


def test_noalloc_matches_regular_entry_point_twice_in_a_row():
    small = synth.plain_512()
    big = synth.production_4096()
    sub = big.ulhc[::37]                      # 390 pairs: more than one refinement chunk
    want_small = run_regular(small, small.ulhc)
    want_big = run_regular(big, sub)
    # two calls in a row with different geometries, then the first one again
    for w, ulhc, want in ((small, small.ulhc, want_small), (big, sub, want_big),
                          (small, small.ulhc, want_small)):
        off, diag = run_noalloc(w, ulhc)
        np.testing.assert_array_equal(off, want[0])
        np.testing.assert_array_equal(diag, want[1])


def test_noalloc_start_up_call_and_bounds():
    # a call with no pairs is the start-up call (loads the device code, launches nothing); a pair
    # whose window leaves its raster gives AMPCOR_E_BOUNDS and NaN offsets for that pair only,
    # and the next clean call returns OK because each call clears the shared bounds counter
    lib = _lib.load()
    w = synth.plain_512()
    err = ctypes.create_string_buffer(256)
    empty = _lib.Job(ref=None, ref_lines=0, ref_samples=0, tgt=None, tgt_lines=0, tgt_samples=0,
                     ulhc=None, pairs=0, offsets=None)
    assert lib.ampcor_correlate_noalloc(ctypes.byref(params_of(w)), ctypes.byref(empty), None, err,
                                        len(err)) == _lib.OK, err.value.decode()
    ulhc = w.ulhc[:4].copy()
    ulhc[2, 2] = 500   # window leaves the 512-line raster
    ref, tgt, u = device_batch(w, ulhc)
    off = torch.zeros((4, 2), dtype=torch.float32, device=ref.device)
    job = _lib.Job(ref=ref.data_ptr(), ref_lines=512, ref_samples=512, tgt=tgt.data_ptr(),
                   tgt_lines=512, tgt_samples=512, ulhc=u.data_ptr(), pairs=4,
                   offsets=off.data_ptr())
    st = ctypes.c_void_p(torch_stream_handle(None, ref.device))
    rc = lib.ampcor_correlate_noalloc(ctypes.byref(params_of(w)), ctypes.byref(job), st, err,
                                      len(err))
    assert rc == _lib.E_BOUNDS and b"leave their raster" in err.value
    o = off.cpu().numpy()
    assert np.isnan(o[2]).all() and np.isfinite(o[[0, 1, 3]]).all()
    got, _ = run_noalloc(w, w.ulhc[:4])
    want, _ = run_regular(w, w.ulhc[:4])
    np.testing.assert_array_equal(got, want)


def test_noalloc_rejects_too_many_pairs():
    lib = _lib.load()
    w = synth.plain_512()
    job = _lib.Job(ref=1, ref_lines=512, ref_samples=512, tgt=1, tgt_lines=512, tgt_samples=512,
                   ulhc=1, pairs=16385, offsets=1)
    err = ctypes.create_string_buffer(256)
    rc = lib.ampcor_correlate_noalloc(ctypes.byref(params_of(w)), ctypes.byref(job), None, err,
                                      len(err))
    assert rc == _lib.E_ARG
    assert b"16384" in err.value
