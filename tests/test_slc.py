"""The SLC file reader (raw row-major complex64, no header; pkg/ampcor/dom/SLC.py semantics)."""
import numpy as np
import pytest

from ampcor_b200.slc import SLC, pixel_size, pinned_empty


def _raster(lines, samples, seed=3):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((lines, samples)) + 1j * rng.standard_normal((lines, samples))).astype(np.complex64)


def test_pixel_size_and_footprint(tmp_path):
    assert pixel_size() == 8
    slc = SLC.write(tmp_path / "a.slc", _raster(5, 7))
    assert slc.shape == (5, 7)
    assert slc.size() == 5 * 7 * 8
    assert (tmp_path / "a.slc").stat().st_size == slc.size()


def test_pixels_by_index_and_offset(tmp_path):
    r = _raster(6, 9)
    slc = SLC.write(tmp_path / "b.slc", r).open()
    assert slc[(2, 3)] == complex(r[2, 3])
    assert slc[2 * 9 + 3] == complex(r[2, 3])
    assert slc[(5, 8)] == complex(r[5, 8])
    with pytest.raises(IndexError):
        slc[(6, 0)]
    with pytest.raises(IndexError):
        slc[6 * 9]


def test_slice_bounds_follow_the_reference(tmp_path):
    # SLC.py: a negative begin or begin + shape past the raster gives no slice
    r = _raster(8, 8)
    slc = SLC.write(tmp_path / "c.slc", r)
    np.testing.assert_array_equal(slc.slice((2, 3), (4, 5)), r[2:6, 3:8])
    np.testing.assert_array_equal(slc.slice((0, 0), (8, 8)), r)
    assert slc.slice((-1, 0), (2, 2)) is None
    assert slc.slice((5, 5), (4, 2)) is None
    assert slc.slice((5, 5), (2, 4)) is None


def test_short_file_and_bad_mode_are_errors(tmp_path):
    SLC.write(tmp_path / "d.slc", _raster(4, 4))
    with pytest.raises(ValueError):
        SLC(tmp_path / "d.slc", (5, 4)).open()
    with pytest.raises(ValueError):
        SLC(tmp_path / "d.slc", (4, 4)).open("w")
    with pytest.raises(ValueError):
        SLC(tmp_path / "d.slc", (0, 4))


def test_pinned_copy_matches_the_file(tmp_path):
    r = _raster(37, 11)
    slc = SLC.write(tmp_path / "e.slc", r)
    p = slc.pinned(rows_per_read=5)
    assert p.shape == r.shape and p.dtype == np.complex64
    np.testing.assert_array_equal(p, r)
    e = pinned_empty((3, 4))
    assert e.shape == (3, 4) and e.dtype == np.complex64


@pytest.mark.gpu
def test_correlation_from_files_matches_arrays(tmp_path):
    # rasters read from SLC files into page-locked memory go through the banded host path and
    # give the offsets of the same rasters passed as arrays
    from ampcor_b200 import synth
    from ampcor_b200.worker import Worker

    w = synth.plain_512()
    ref = SLC.write(tmp_path / "ref.slc", w.ref).pinned()
    tgt = SLC.write(tmp_path / "tgt.slc", w.tgt).pinned()
    worker = Worker(pairs=w.pairs, chip=(32, 32), window=(48, 48), refine_factor=2,
                    refine_margin=4, zoom_factor=4)
    from_files = worker.correlate(ref, tgt, w.ulhc)
    from_arrays = worker.correlate(w.ref, w.tgt, w.ulhc)
    worker.close()
    assert np.array_equal(from_files, from_arrays)
