"""Row-band sharding across ranks and the final offset gather, with two gloo ranks on CPU.

Each rank correlates its own band (here with the FP64 oracle standing in for the GPU, since this
runs without one) and the gathered field must equal the single-rank result pair for pair.
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
