"""The oracle against the known answers of the reference's own tests (CPU only).

Every check names the reference test it restates.  These pin the oracle before it is used as
the checker of the CUDA path.
"""
import numpy as np
import pytest

import oracle
from oracle import npref
from ampcor_b200 import synth
from ampcor_b200.worker import DIAG_DTYPE

from fixtures import placement_identity


def test_sat_of_ones():
    # tests/libampcor/sumarea.cc:28-58: the SAT of a grid of ones is (i+1)(j+1)
    s = oracle.sat(np.ones((7, 5)))
    i, j = np.indices((7, 5))
    assert np.array_equal(s, (i + 1.0) * (j + 1.0))


def test_sat_box_sums():
    # tests/libampcor/sumarea-sum.cc:28-144: whole grid, interior, left column, top row
    rows, cols = 9, 6
    s = oracle.sat(np.ones((rows, cols)))
    assert oracle.box(s, 0, 0, rows, cols) == rows * cols
    assert oracle.box(s, 1, 1, rows - 1, cols - 1) == (rows - 2) * (cols - 2)
    assert oracle.box(s, 0, 0, rows, 1) == rows
    assert oracle.box(s, 0, 0, 1, cols) == cols


def test_sat_matches_direct_sums():
    # tests/cuda/tile-sat.cu:254-265: SAT against a host gold, exact for integers
    rng = np.random.default_rng(1)
    x = rng.integers(0, 100, (16, 16)).astype(np.float64)
    s = oracle.sat(x)
    assert np.array_equal(s, x.cumsum(0).cumsum(1))


def test_window_means_match_direct():
    # tests/libampcor_cuda/tgtStats.cc:327-365: every placement mean from the SAT equals the
    # direct mean of the placement (R = 64, M = 8 as the reference test)
    R, M = 64, 8
    rng = np.random.default_rng(2)
    win = np.abs(rng.standard_normal((R + 2 * M, R + 2 * M)))
    s = oracle.sat(win)
    for u in range(0, 2 * M + 1, 4):
        for v in range(0, 2 * M + 1, 3):
            direct = win[u:u + R, v:v + R].mean()
            assert oracle.box(s, u, v, u + R, v + R) / R**2 == pytest.approx(direct, rel=1e-13)


def test_chip_stats():
    # tests/libampcor_cuda/refStats.cc:265-313: after mean removal the chip has zero mean and
    # sigma is the root of the sum of squares
    rng = np.random.default_rng(3)
    chip = np.abs(rng.standard_normal((32, 32)))
    win = np.abs(rng.standard_normal((48, 48)))
    _, sigma = oracle.ncc(chip, win)
    assert sigma == pytest.approx(np.sqrt(((chip - chip.mean()) ** 2).sum()), rel=1e-14)


@pytest.mark.parametrize("R,M", [(16, 4), (32, 8)])
def test_placement_identity(R, M):
    # tests/libampcor_cuda/correlate.cc:279-303 (gamma = 1 at the true placement) and
    # maxcor.cc:296-312 (the argmax is the placement); nudge.cc:204-225 (corner bounds)
    ref, tgt, ulhc = placement_identity(R, M, seed=4)
    W, C = R + 2 * M, 2 * M + 1
    chip = np.abs(ref).astype(np.float64)
    for pid in range(0, C * C, 7):
        i, j = divmod(pid, C)
        win = np.abs(tgt[pid * W:(pid + 1) * W]).astype(np.float64)
        g, _ = oracle.ncc(chip, win)
        assert g[i, j] == pytest.approx(1.0, abs=1e-12)
        k = oracle.argmax_first(g)
        assert divmod(k, C) == (i, j)
        for m in (2, 4, M):
            top, left = oracle.nudge(i, j, R, W, m)
            assert 0 <= top <= W - (R + 2 * m) and 0 <= left <= W - (R + 2 * m)
    arg, gap = oracle.coarse_cpu(ref, tgt, ulhc, R, W)
    assert np.array_equal(arg, np.stack(np.divmod(np.arange(C * C), C), 1))


def test_numerator_closed_form():
    # tests/cuda/tile-correlate.cu:361-373: an all-ones chip against a window whose R x R
    # interior is ones has numerator (R - |M - r|)(R - |M - c|)
    R, M = 16, 5
    chip = np.ones((R, R))
    win = np.zeros((R + 2 * M, R + 2 * M))
    win[M:M + R, M:M + R] = 1.0
    x = oracle.xcorr(chip, win)
    r, c = np.indices(x.shape)
    assert np.array_equal(x, (R - np.abs(M - r)) * (R - np.abs(M - c)))


def test_fft_of_constant_is_delta():
    # tests/cuda/tile-refine.cu:367-400: the transform of a constant quadrant is a delta at the
    # origin; hence band-limited upsampling reproduces a constant exactly
    dim = 16
    q = np.full((dim // 2, dim // 2), 0.5 + 0j)
    F = np.fft.fft2(q)
    assert F[0, 0] != 0 and np.count_nonzero(np.abs(F) > 1e-12) == 1
    up = oracle.upsample(q, 2)
    assert np.allclose(up, 0.5, atol=1e-14)


@pytest.mark.parametrize("N,f", [(8, 2), (9, 3), (32, 2), (40, 2), (64, 2), (80, 2)])
def test_upsample_matches_numpy_fft(N, f):
    rng = np.random.default_rng(N * f)
    t = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    a = oracle.upsample(t, f)
    b = npref.upsample_fft(t, f)
    assert np.abs(a - b).max() < 1e-12
    assert np.array_equal(a[::f, ::f], t)   # interpolation keeps the samples


@pytest.mark.parametrize("Cf,z", [(17, 4), (33, 8)])
def test_zoom_matches_numpy_fft(Cf, z):
    rng = np.random.default_rng(Cf)
    G = rng.standard_normal((Cf, Cf))
    assert np.abs(oracle.zoom(G, z) - npref.zoom_fft(G, z)).max() < 1e-12
    assert np.abs(oracle.zoom(G, z, use_abs=True) - npref.zoom_fft(G, z, use_abs=True)).max() < 1e-12


def test_plain_512_offsets():
    # the CPU-runnable configuration: every pair sees the same (+3.4, -2.7) px shift, the
    # sub-pixel quantum is 1/8 px, so the answer is the nearest grid point (3.375, -2.75)
    w = synth.plain_512()
    off, diag = oracle.adjust(w.ref, w.tgt, w.ulhc, 32, 48, 2, 4, 4)
    assert w.pairs == 64
    assert np.all(off == np.float32([3.375, -2.75]))
    # the reference CPU correlator picks the same integer offsets
    arg, gap = oracle.coarse_cpu(w.ref, w.tgt, w.ulhc, 32, 48)
    assert np.array_equal(arg[:, 0], diag["coarse_u"]) and np.array_equal(arg[:, 1], diag["coarse_v"])
    assert np.all(arg == [11, 5])   # M + round(3.4), M + round(-2.7)


def test_ref_compat_offsets_subtract_margin_again():
    # offsets.cu:124-125 subtracts the refine margin from the nudged corner a second time
    w = synth.plain_512()
    off, _ = oracle.adjust(w.ref, w.tgt, w.ulhc[:4], 32, 48, 2, 4, 4)
    off_c, _ = oracle.adjust(w.ref, w.tgt, w.ulhc[:4], 32, 48, 2, 4, 4, ref_compat=True)
    assert np.allclose(off_c, off - 4)


def test_golden_plain_512():
    # regression pin of the oracle on the CPU-runnable configuration (tests/golden/make_golden.py)
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "plain_512.npz"))
    w = synth.plain_512()
    assert np.array_equal(g["ulhc"], w.ulhc)
    off, diag = oracle.adjust(w.ref, w.tgt, w.ulhc, 32, 48, 2, 4, 4)
    assert np.array_equal(off, g["offsets"])
    assert np.allclose(diag["refined_peak"], g["refined_peak"], rtol=1e-12, atol=0)
    assert np.array_equal(diag["fine_p"], g["fine_p"]) and np.array_equal(diag["fine_q"], g["fine_q"])


def test_oracle_deramp_tile():
    # a smooth field under a linear phase ramp: the deramp keeps every amplitude and leaves no
    # phase step along lines or samples
    n = 16
    y, x = np.mgrid[0:n, 0:n]
    rng = np.random.default_rng(0)
    F = np.fft.fft2(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    F[4:-4, :] = 0
    F[:, 4:-4] = 0
    t = np.fft.ifft2(F) * np.exp(1j * (0.9 * x + 0.4 * y))
    d = oracle.deramp(t)
    np.testing.assert_allclose(np.abs(d), np.abs(t), atol=1e-12)
    assert abs(np.angle((d[:, 1:] * np.conj(d[:, :-1])).sum())) < 1e-12
    assert abs(np.angle((d[1:, :] * np.conj(d[:-1, :])).sum())) < 1e-12


def test_oracle_deramp_restores_doppler_offsets():
    # speckle off baseband: the zero-padded refinement alone misplaces the sub-pixel offsets, the
    # deramp before it restores them to the zoom grid's rounding of the applied shift
    from ampcor_b200 import synth

    w = synth.doppler_512()
    plain, _ = oracle.adjust(w.ref, w.tgt, w.ulhc, 32, 48, 2, 4, 4)
    deramped, _ = oracle.adjust(w.ref, w.tgt, w.ulhc, 32, 48, 2, 4, 4, deramp=True)
    quantum = 1.0 / 8
    assert np.abs(plain - w.truth).mean() > 0.15
    assert np.abs(deramped - w.truth).max() <= quantum / 2 + 1e-6
    flat = synth.doppler_512(ramp=(0.0, 0.0))
    a, _ = oracle.adjust(flat.ref, flat.tgt, flat.ulhc, 32, 48, 2, 4, 4)
    assert np.array_equal(deramped, a)


def test_parity_checker_rules():
    # the pair-by-pair checker on CPU: the oracle's own results (as float32) pass with nothing
    # excused; a coarse cell moved on a pair with a clear maximum fails; moving the cell of the
    # pair with the smallest top-two gap is excused when its surface error explains the gap
    from oracle import parity

    w = synth.plain_512()
    orc = parity.oracle_run(w.ref, w.tgt, w.ulhc, 32, 48, 2, 4, 4)
    od = orc["diag"]
    gd = np.zeros(len(od), dtype=DIAG_DTYPE)
    for k in ("coarse_u", "coarse_v", "top", "left", "fine_p", "fine_q"):
        gd[k] = od[k]
    gd["refined_peak"] = od["refined_peak"]
    gd["coarse_peak"] = od["coarse_peak"]
    cs = orc["coarse"].astype(np.float32)
    rs = orc["refined"].astype(np.float32)
    rep = parity.compare(orc, orc["offsets"], gd, cs, rs)
    assert rep["failures"] == [] and rep["pairs_excused"] == 0 and rep["pairs_checked"] == 64
    assert rep["max_abs_err_vs_oracle_px"] == 0.0
    bad = gd.copy()
    bad["coarse_v"][5] += 1
    rep = parity.compare(orc, orc["offsets"], bad, cs, rs)
    assert [f[0] for f in rep["failures"]][:1] == [5]
    # a near-tie: make pair p's second-best coarse cell win, with a surface error that covers it
    p = int(np.argmin(od["coarse_gap"]))
    C = 17
    surf = orc["coarse"][p].reshape(-1)
    k2 = int(np.argsort(surf)[-2])
    tie = gd.copy()
    tie["coarse_u"][p], tie["coarse_v"][p] = divmod(k2, C)
    cs2 = cs.copy()
    cs2[p].reshape(-1)[k2] += np.float32(od["coarse_gap"][p])
    rep = parity.compare(orc, orc["offsets"], tie, cs2, rs)
    coarse_fail = [f for f in rep["failures"] if "coarse cell" in f[1]]
    assert coarse_fail == [] and rep["coarse_cells_differing"] == 1
