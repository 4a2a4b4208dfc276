"""The FP64 oracle pinned to the reference's own CPU code (CPU only).

``oracle/_ref/libampcor_ref.so`` is the reference's CPU correlator (lib/libampcor/correlators/
Sequential.cc, Sequential.icc, SumArea.icc) and SLC raster (lib/libampcor/dom/SLC.icc), compiled
unmodified from the reference tree against stand-ins of pyre (``oracle/ref_shim``), driven
through the reference's own addReferenceTile / addTargetTile / adjust.  These tests need that
library (``make -C oracle`` where the reference source tree is present) and skip without it.

What they pin:

* ``oracle.coarse_cpu(as_built=True)`` reproduces the reference's correlation surfaces bit for bit;
  as written, the reference's summed-area table is built over a new grid of the window's layout
  (Sequential.cc:48), not over the window, so its box means are zero and its surface is the
  uncentred ratio sum a_r t / sqrt(sum a_r^2 sum t^2);
* the reference's SumArea, given the window amplitudes, gives the oracle's summed-area table and
  box sums, the step the default (intended) ``oracle.coarse_cpu`` adds; so every step of the
  integer-offset gate is the reference's own arithmetic, with the table built from the window;
* on the reference's own configurations the as-built and the intended correlators agree on the
  integer offsets of every pair whose as-built top-two gap is clear.
"""
import numpy as np
import pytest

import oracle
from oracle import ref as refcpu
from ampcor_b200 import synth

from fixtures import placement_identity

pytestmark = pytest.mark.skipif(not refcpu.available(),
                                reason="the reference's CPU correlator is not built (no reference tree)")


def _surfaces(w, ulhc, R, W, threads=4):
    with refcpu.Rasters(w.ref, w.tgt) as r:
        return refcpu.sequential(r, ulhc, R, W, threads=threads)


def test_as_built_restatement_is_the_reference_bit_for_bit():
    w = synth.plain_512()
    got = _surfaces(w, w.ulhc, 32, 48)
    _, _, want = oracle.coarse_cpu(w.ref, w.tgt, w.ulhc, 32, 48, surfaces=True, as_built=True)
    np.testing.assert_array_equal(got, want)
    # production geometry (64^2 chips, +-32 px) and its heavy-tailed variant, spread-out pairs
    for heavy in (False, True):
        w = synth.production_4096(heavy_tail=heavy)
        idx = np.linspace(0, w.pairs - 1, 12).round().astype(int)
        got = _surfaces(w, w.ulhc[idx], 64, 128)
        _, _, want = oracle.coarse_cpu(w.ref, w.tgt, w.ulhc[idx], 64, 128, surfaces=True,
                                       as_built=True)
        np.testing.assert_array_equal(got, want)


def test_as_built_reference_on_the_placement_identity_fixture():
    # tests/libampcor_cuda/correlate.cc:119-143: the chip pasted into an otherwise zero window;
    # the as-built surface is 1 at the placement too (no mean is taken off either tile), and
    # placements whose box is all zero divide zero by zero in the reference and here alike
    ref, tgt, ulhc = placement_identity(32, 8, seed=5)

    class W:
        pass

    w = W()
    w.ref, w.tgt = ref, tgt
    got = _surfaces(w, ulhc, 32, 48)
    _, _, want = oracle.coarse_cpu(ref, tgt, ulhc, 32, 48, surfaces=True, as_built=True)
    np.testing.assert_array_equal(got, want)
    C = 17
    i, j = np.divmod(np.arange(C * C), C)
    np.testing.assert_allclose(got[np.arange(C * C), i, j], 1.0, rtol=1e-12)


def test_reference_sumarea_is_the_oracle_table():
    # tests/libampcor/sumarea.cc: a grid of ones gives (i + 1)(j + 1)
    table, _ = refcpu.sumarea(np.ones((5, 5)))
    i, j = np.mgrid[0:5, 0:5]
    np.testing.assert_array_equal(table, (i + 1.0) * (j + 1.0))
    # window amplitudes of a production pair: the same table and box sums as the oracle's
    w = synth.production_4096()
    l, s = w.ulhc[777, 2:]
    a = np.abs(w.tgt[l:l + 128, s:s + 128]).astype(np.float64)
    rng = np.random.default_rng(4)
    boxes = [(int(u), int(v), 64, 64) for u, v in rng.integers(0, 65, size=(40, 2))]
    boxes += [(0, 0, 64, 64), (64, 64, 64, 64), (0, 64, 64, 64)]
    table, sums = refcpu.sumarea(a, boxes)
    mine = oracle.sat(a)
    np.testing.assert_allclose(table, mine, rtol=1e-15, atol=0)
    for (u, v, hh, ww), got in zip(boxes, sums):
        want = oracle.box(mine, u, v, u + hh, v + ww)
        assert got == pytest.approx(want, rel=1e-12, abs=1e-9)
        assert got == pytest.approx(a[u:u + hh, v:v + ww].sum(), rel=1e-12)


def test_as_built_and_intended_integer_offsets_agree_where_clear():
    # the two correlators differ in value (no mean removal as built) but, on speckle, not in the
    # integer offset of any pair whose as-built maximum is clear of its runner-up
    for w, R, W, idx in ((synth.plain_512(), 32, 48, None),
                         (synth.production_4096(), 64, 128, np.arange(0, 14400, 1200))):
        ulhc = w.ulhc if idx is None else w.ulhc[idx]
        built = _surfaces(w, ulhc, R, W)
        arg, _ = oracle.coarse_cpu(w.ref, w.tgt, ulhc, R, W)
        C = W - R + 1
        flat = built.reshape(len(ulhc), -1)
        k = flat.argmax(axis=1)
        top2 = np.sort(flat, axis=1)[:, -2:]
        clear = (top2[:, 1] - top2[:, 0]) > 1e-9
        assert np.array_equal(k[clear], (arg[:, 0] * C + arg[:, 1])[clear])
