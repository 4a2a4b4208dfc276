"""Multi-GPU sharding of a correlation job (one process per GPU).

Tile pairs are independent (the reference worker has no cross-pair step,
lib/libampcor_cuda/correlators/Sequential.icc:47-141), so a job splits into contiguous row bands
of tile centres, one band per rank, with no collective on the data path.  Each rank needs only
the raster lines its band touches (:func:`band_lines`), so a rank can copy just that slab into its
own HBM.  The only exchange is the final gather of the offset field (8 bytes per pair).
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
