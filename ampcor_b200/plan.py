"""Tile-pair planning with the semantics of ampcor's pyre components.

* :func:`uniform_grid` - tile centres of ``UniformGrid.points`` (pkg/ampcor/correlators/
  UniformGrid.py:34-54);
* :func:`constant_codomain` - the ``Constant`` coarse map (Constant.py:32-43);
* :func:`plan_pairs` - ``Plan.assemble`` (Plan.py:143-185): reference chip corner
  ``p - chip//2``, search window corner ``q - chip//2 - padding``, a pair kept only when both
  slices lie inside their rasters (SLC.slice, pkg/ampcor/dom/SLC.py:54-76).
"""
from __future__ import annotations

import itertools

import numpy as np


def uniform_grid(bounds, shape):
    """Centres of a ``shape`` grid of tiles evenly spaced over a raster of ``bounds``."""
    tile = tuple(b // s for b, s in zip(bounds, shape))
    margin = tuple(b % s for b, s in zip(bounds, shape))
    ticks = tuple(
        tuple(m // 2 + n * t + t // 2 for n in range(g)) for g, m, t in zip(shape, margin, tile)
    )
    return tuple(itertools.product(*ticks))


def constant_codomain(domain, shift=(0, 0)):
    """Images of ``domain`` under a constant shift."""
    return tuple(tuple(p + s for p, s in zip(point, shift)) for point in domain)


def _valid(begin, shape, bounds):
    return all(b >= 0 for b in begin) and all(b + s <= l for b, s, l in zip(begin, shape, bounds))


def plan_pairs(domain, codomain, chip, padding, ref_shape, tgt_shape):
    """Corners of the valid tile pairs.

    Returns ``(ulhc, valid)``: ``ulhc`` is an int32 array (valid pairs x 4) of chip line, chip
    sample, window line, window sample, in grid order with invalid pairs dropped (the compacted
    pair index of ``Plan.pairs``); ``valid`` is the boolean mask over the grid points.
    """
    chip = tuple(int(c) for c in chip)
    padding = tuple(int(p) for p in padding)
    window = tuple(c + 2 * p for c, p in zip(chip, padding))
    rows, mask = [], []
    for ref, tgt in zip(domain, codomain):
        rb = tuple(r - c // 2 for r, c in zip(ref, chip))
        tb = tuple(t - c // 2 - p for t, c, p in zip(tgt, chip, padding))
        ok = _valid(rb, chip, ref_shape) and _valid(tb, window, tgt_shape)
        mask.append(ok)
        if ok:
            rows.append((rb[0], rb[1], tb[0], tb[1]))
    ulhc = np.asarray(rows, dtype=np.int32).reshape(-1, 4)
    return ulhc, np.asarray(mask, dtype=bool)
