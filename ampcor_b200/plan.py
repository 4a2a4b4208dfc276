"""Tile-pair planning with the semantics of ampcor's pyre components.

* :func:`uniform_grid` - tile centres of ``UniformGrid.points`` (pkg/ampcor/correlators/
  UniformGrid.py:34-54);
* :func:`constant_codomain` - the ``Constant`` coarse map (Constant.py:32-43);
* :func:`plan_pairs` - ``Plan.assemble`` (Plan.py:143-185): reference chip corner
  ``p - chip//2``, search window corner ``q - chip//2 - padding``, a pair kept only when both
  slices lie inside their rasters (SLC.slice, pkg/ampcor/dom/SLC.py:54-76);
* :class:`OffsetMap` - the map of reference points to target points on the grid of tiles
  (pkg/ampcor/dom/OffsetMap.py:14-95), built as the coarse map by :func:`coarse_map`
  (``Grid.map``, pkg/ampcor/correlators/Grid.py:34-50) and, after a correlation, refined by
  :func:`refined_map`, which moves each valid pair's target point by its offset.
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


class OffsetMap:
    """Reference points (``domain``) and their target points (``codomain``) on a logically
    Cartesian grid of ``shape`` (pkg/ampcor/dom/OffsetMap.py:14-95).  ``layout`` is the packing
    order of the grid axes, fastest first; the default is row-major, the order in which
    :func:`uniform_grid` lists its points.  Indexing by a grid index returns ``(ref, tgt)``."""

    def __init__(self, shape, layout=None):
        self.shape = tuple(int(s) for s in shape)
        self.layout = tuple(layout) if layout is not None else tuple(reversed(range(len(self.shape))))
        if sorted(self.layout) != list(range(len(self.shape))):
            raise ValueError(f"layout {self.layout} is not a permutation of the axes")
        self.domain = [None] * self.size
        self.codomain = [None] * self.size

    @property
    def size(self):
        return int(np.prod(self.shape)) if self.shape else 0

    def __len__(self):
        return self.size

    def offset(self, index):
        """Position of grid ``index`` in the domain / codomain sequences."""
        if len(index) != len(self.shape) or any(not 0 <= i < n for i, n in zip(index, self.shape)):
            raise IndexError(f"index {tuple(index)} outside a grid of shape {self.shape}")
        off, stride = 0, 1
        for axis in self.layout:
            off += int(index[axis]) * stride
            stride *= self.shape[axis]
        return off

    def index(self, offset):
        """The grid index stored at position ``offset``."""
        idx = [0] * len(self.shape)
        for axis in self.layout:
            offset, idx[axis] = divmod(int(offset), self.shape[axis])
        return tuple(idx)

    def __getitem__(self, index):
        k = self.offset(index)
        return self.domain[k], self.codomain[k]

    def __setitem__(self, index, points):
        k = self.offset(index)
        self.domain[k], self.codomain[k] = points

    def field(self):
        """The offset field: a (*shape, 2) float32 array of ``tgt - ref`` per grid point, NaN
        where the map has no target point (pairs the plan dropped or whose tiles left a raster)."""
        out = np.full(self.shape + (2,), np.nan, np.float32)
        for k in range(self.size):
            ref, tgt = self.domain[k], self.codomain[k]
            if ref is not None and tgt is not None:
                out[self.index(k)] = np.subtract(tgt, ref, dtype=np.float64)
        return out


def coarse_map(shape, bounds, shift=(0, 0)):
    """The coarse offset map of ``Grid.map`` (Grid.py:34-50) with a ``Constant`` functor: a
    ``shape`` grid of points over a raster of ``bounds`` (:func:`uniform_grid`), each mapped to
    itself plus ``shift``."""
    omap = OffsetMap(shape)
    omap.domain = list(uniform_grid(bounds, shape))
    omap.codomain = list(constant_codomain(omap.domain, shift))
    return omap


def refined_map(coarse, valid, offsets):
    """The refined offset map of a correlation: grid point k of ``coarse`` with
    ``valid[k]`` (the mask of :func:`plan_pairs`) took pair ``j`` (its rank among the valid
    points, the compacted pair index of ``Plan.pairs``), and its target point moves by
    ``offsets[j]`` = (dy, dx).  Points the plan dropped, and pairs whose offsets are NaN, get no
    target point."""
    valid = np.asarray(valid, bool).reshape(-1)
    offsets = np.asarray(offsets, np.float64).reshape(-1, 2)
    if valid.size != coarse.size:
        raise ValueError("the validity mask must cover every point of the coarse map")
    if offsets.shape[0] != int(valid.sum()):
        raise ValueError("one offset pair per valid tile pair")
    out = OffsetMap(coarse.shape, coarse.layout)
    out.domain = list(coarse.domain)
    pair = np.cumsum(valid) - 1
    for k in range(coarse.size):
        if valid[k] and np.isfinite(offsets[pair[k]]).all():
            out.codomain[k] = tuple(float(c) + float(d) for c, d in zip(coarse.codomain[k], offsets[pair[k]]))
    return out
