"""Multi-GPU sharding of a correlation job (one process per GPU).

Tile pairs are independent (the reference worker has no cross-pair step,
lib/libampcor_cuda/correlators/Sequential.icc:47-141), so a job splits into contiguous row bands
of tile centres, one band per rank, with no collective on the data path.  Each rank needs only
the raster lines its band touches (:func:`band_lines`), so a rank can copy just that slab into its
own HBM.  The only exchange is the final gather of the offset field (8 bytes per pair).
:func:`correlate_sharded` puts the pieces together for one job.
"""
from __future__ import annotations

import numpy as np


def shard(ulhc, rank, world):
    """Indices of the pairs of ``rank``: contiguous row bands of the pairs ordered by chip line
    (ties by sample), balanced to within one pair."""
    ulhc = np.asarray(ulhc).reshape(-1, 4)
    order = np.lexsort((ulhc[:, 1], ulhc[:, 0]))
    bounds = np.linspace(0, len(order), world + 1).round().astype(int)
    return np.sort(order[bounds[rank]:bounds[rank + 1]])


def band_lines(ulhc, chip, window):
    """[first, last) raster lines of the reference and secondary rasters that a set of pairs reads."""
    ulhc = np.asarray(ulhc).reshape(-1, 4)
    if len(ulhc) == 0:
        return (0, 0), (0, 0)
    return ((int(ulhc[:, 0].min()), int(ulhc[:, 0].max()) + chip),
            (int(ulhc[:, 2].min()), int(ulhc[:, 2].max()) + window))


def gather_offsets(local_offsets, local_index, total, group=None):
    """All-gather the per-rank offsets (float32, pairs x 2) into the full field in pair order."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    n = torch.tensor([len(local_index)], dtype=torch.int64)
    counts = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(counts, n, group=group)
    cap = int(max(c.item() for c in counts))
    idx = torch.full((cap,), -1, dtype=torch.int64)
    idx[: len(local_index)] = torch.as_tensor(np.asarray(local_index), dtype=torch.int64)
    off = torch.zeros((cap, 2), dtype=torch.float32)
    off[: len(local_index)] = torch.as_tensor(np.asarray(local_offsets), dtype=torch.float32)
    all_idx = [torch.empty_like(idx) for _ in range(world)]
    all_off = [torch.empty_like(off) for _ in range(world)]
    dist.all_gather(all_idx, idx, group=group)
    dist.all_gather(all_off, off, group=group)
    full = np.full((total, 2), np.nan, np.float32)
    for i, o in zip(all_idx, all_off):
        keep = i >= 0
        full[i[keep].numpy()] = o[keep].numpy()
    return full


def band(ref, tgt, ulhc, chip, window, rank, world):
    """The slice of one job that ``rank`` correlates: its pair indices, the raster lines its
    pairs read (reference and secondary, as views of the full rasters) and its corners rebased to
    those lines."""
    ulhc = np.asarray(ulhc).reshape(-1, 4)
    idx = shard(ulhc, rank, world)
    (r0, r1), (t0, t1) = band_lines(ulhc[idx], chip, window)
    local = ulhc[idx].astype(np.int64) - np.array([r0, 0, t0, 0], np.int64)
    return idx, ref[r0:r1], tgt[t0:t1], np.ascontiguousarray(local, np.int32)


def correlate_sharded(correlate, ref, tgt, ulhc, chip, window, group=None):
    """Correlate one job over the ranks of ``group``: each rank takes its row band of pairs,
    hands ``correlate(ref_band, tgt_band, ulhc_band)`` only the raster lines that band reads (so a
    worker's host path uploads just those), and the offsets are gathered into the full field in
    pair order on every rank.  ``correlate`` is typically ``Worker.correlate`` with host rasters."""
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    idx, ref_b, tgt_b, local = band(ref, tgt, ulhc, chip, window, rank, world)
    if len(idx):
        off = np.asarray(correlate(np.ascontiguousarray(ref_b), np.ascontiguousarray(tgt_b), local),
                         np.float32).reshape(-1, 2)
    else:
        off = np.zeros((0, 2), np.float32)
    return gather_offsets(off, idx, len(np.asarray(ulhc).reshape(-1, 4)), group=group)
