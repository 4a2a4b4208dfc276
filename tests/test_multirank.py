"""Row-band sharding across ranks and the final offset gather, with two gloo ranks on CPU.

Each rank correlates its own band (here with the FP64 oracle standing in for the GPU, since this
runs without one) and the gathered field must equal the single-rank result pair for pair.  Through
parallel.correlate_sharded a rank sees only the raster lines its band reads, with its corners
rebased to them.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ampcor_b200 import parallel, synth


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w = synth.plain_512()
        idx = parallel.shard(w.ulhc, rank, world)
        off, _ = oracle.adjust(w.ref, w.tgt, w.ulhc[idx], 32, 48, 2, 4, 4, threads=1)
        full = parallel.gather_offsets(off, idx, w.pairs)
        if rank == 0:
            np.save(out, full)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _band_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w = synth.production_4096()
        sub = w.ulhc[::97]
        seen = {}

        def correlate(ref_b, tgt_b, ulhc_b):
            seen["lines"] = (ref_b.shape[0], tgt_b.shape[0])
            off, _ = oracle.adjust(ref_b, tgt_b, ulhc_b, 64, 128, 2, 8, 8, threads=2)
            return off

        full = parallel.correlate_sharded(correlate, w.ref, w.tgt, sub, 64, 128)
        np.save(f"{out}.{rank}.npy", full)
        np.save(f"{out}.lines{rank}.npy", np.array(seen["lines"]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_correlate_sharded_uploads_bands_and_matches_one_rank(tmp_path):
    import oracle

    out = str(tmp_path / "field")
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_band_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    w = synth.production_4096()
    sub = w.ulhc[::97]
    want, _ = oracle.adjust(w.ref, w.tgt, sub, 64, 128, 2, 8, 8)
    for r in range(2):
        assert np.array_equal(np.load(f"{out}.{r}.npy"), want)
        ref_lines, tgt_lines = np.load(f"{out}.lines{r}.npy")
        assert ref_lines < 4096 * 0.6 and tgt_lines < 4096 * 0.6  # a band, not the raster
    # the rebased corners address the same pixels as the original ones
    for r in range(2):
        idx, ref_b, tgt_b, local = parallel.band(w.ref, w.tgt, sub, 64, 128, r, 2)
        for k in (0, len(idx) - 1):
            a, b, c, d = local[k]
            A, B, Cc, D = sub[idx[k]]
            assert np.array_equal(ref_b[a:a + 64, b:b + 64], w.ref[A:A + 64, B:B + 64])
            assert np.array_equal(tgt_b[c:c + 128, d:d + 128], w.tgt[Cc:Cc + 128, D:D + 128])


def test_shards_partition_the_pairs():
    w = synth.plain_512()
    parts = [parallel.shard(w.ulhc, r, 3) for r in range(3)]
    allidx = np.concatenate(parts)
    assert sorted(allidx.tolist()) == list(range(w.pairs))
    assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
    # bands are contiguous in chip line: no line range of a rank starts before the previous ends
    firsts = [w.ulhc[p, 0].min() for p in parts]
    lasts = [w.ulhc[p, 0].max() for p in parts]
    assert all(lasts[r] <= firsts[r + 1] for r in range(2))
    (r0, r1), (t0, t1) = parallel.band_lines(w.ulhc[parts[0]], 32, 48)
    assert r0 == w.ulhc[parts[0], 0].min() and r1 == w.ulhc[parts[0], 0].max() + 32


def test_two_gloo_ranks_match_one(tmp_path):
    import oracle

    out = str(tmp_path / "full.npy")
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    w = synth.plain_512()
    want, _ = oracle.adjust(w.ref, w.tgt, w.ulhc, 32, 48, 2, 4, 4)
    assert np.array_equal(np.load(out), want)
