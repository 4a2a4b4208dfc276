"""Restated fixtures of the reference's stage tests.

placement_identity(R, M, seed): the fixture of tests/libampcor_cuda/correlate.cc:119-143 (and
maxcor.cc, tgtStats.cc, nudge.cc): one random-normal real chip; (2M+1)^2 pairs, pair (i, j)
has an all-zero (R+2M)^2 window with the chip pasted at (i, j).  The reference seeds from
std::random_device; here the seed is fixed.  Returned as rasters + corners so the same data
feeds the oracle and the CUDA path: the chip raster is R x R; the window raster stacks the
(2M+1)^2 windows vertically.
"""
import numpy as np


def placement_identity(R, M, seed=0, step=1):
    """``step`` > 1 keeps every step-th placement along each axis (plus the last), for the large
    margins whose full fixture would hold (2M+1)^2 windows; the placements of the returned pairs
    are ``placements`` (pairs x 2)."""
    W = R + 2 * M
    C = 2 * M + 1
    rng = np.random.default_rng(seed)
    chip = rng.standard_normal((R, R)).astype(np.float32)
    ref = chip.astype(np.complex64)
    axis = sorted(set(range(0, C, step)) | {C - 1})
    cells = [(i, j) for i in axis for j in axis]
    pairs = len(cells)
    tgt = np.zeros((pairs * W, W), np.complex64)
    ulhc = np.zeros((pairs, 4), np.int32)
    for pid, (i, j) in enumerate(cells):
        tgt[pid * W + i: pid * W + i + R, j: j + R] = chip
        ulhc[pid] = (0, 0, pid * W, 0)
    if step == 1:
        return ref, tgt, ulhc
    return ref, tgt, ulhc, np.asarray(cells, np.int32)
