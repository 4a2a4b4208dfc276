"""Autotuner of the correlator.

For one worker geometry (chip, window, refinement and zoom) it times every candidate
configuration - correlation form (spectral, bf16x3 tensor-core or plain FP32) x refinement chunk
(pairs per pass of the pipeline: larger chunks mean fewer launches and whole waves, smaller ones
keep more of the refine -> fine hand-off in L2) - on the caller's own device-resident batch and
keeps the fastest.  Results are cached per device name and
geometry in a JSON file (``AMPCOR_TUNE_CACHE``, default ``~/.cache/ampcor_b200/tune.json``).
"""
from __future__ import annotations

import json
import os

DEFAULT_CHUNKS = (296, 592, 1184, 2368, 4736, 9472, 18944)


def _cache_path():
    return os.environ.get("AMPCOR_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "ampcor_b200", "tune.json"))


def _key(worker, device_name):
    return (f"{device_name}|chip{worker.chip[0]}|win{worker.window[0]}|f{worker.refine_factor}"
            f"|m{worker.refine_margin}|z{worker.zoom_factor}")


def _load():
    try:
        with open(_cache_path()) as fh:
            return json.load(fh)
    except Exception:
        return {}


def _store(table):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp"
        with open(tmp, "w") as fh:
            json.dump(table, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def tune(worker, ref, tgt, ulhc, forms=("spectral", "tensor", "plain"), chunks=DEFAULT_CHUNKS, reps=2,
         use_cache=True):
    """Configure ``worker`` with the fastest (form, chunk) for this batch; returns the choice
    with the timings of every candidate (ms per batch)."""
    import torch

    from .worker import Error

    name = torch.cuda.get_device_name(ref.device)
    key = _key(worker, name)
    table = _load() if use_cache else {}
    if use_cache and key in table:
        choice = table[key]
        worker.configure(choice["form"], choice["chunk"])
        return dict(choice, cached=True)
    out = torch.empty((ulhc.shape[0], 2), dtype=torch.float32, device=ref.device)
    results = []
    pairs = int(ulhc.shape[0])
    for form in forms:
        whole = False  # a chunk of at least the whole batch has been timed for this form
        for chunk in sorted(chunks):
            if chunk >= pairs:
                if whole:
                    continue
                whole = True
            try:
                worker.configure(form, chunk)
            except Error:
                continue
            if worker.form != form:
                continue
            try:
                worker.correlate(ref, tgt, ulhc, offsets=out, synchronize=True)
            except Error:
                continue  # e.g. the chunk's scratch does not fit beside the caller's data
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                worker.correlate(ref, tgt, ulhc, offsets=out, synchronize=False)
            e1.record()
            torch.cuda.synchronize()
            results.append({"form": form, "chunk": chunk, "ms": e0.elapsed_time(e1) / reps})
    if not results:
        raise RuntimeError("no configuration of this geometry could run")
    best = min(results, key=lambda r: r["ms"])
    worker.configure(best["form"], best["chunk"])
    choice = {"form": best["form"], "chunk": best["chunk"], "ms": best["ms"], "candidates": results}
    if use_cache:
        table[key] = choice
        _store(table)
    return dict(choice, cached=False)
