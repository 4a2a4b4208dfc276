"""Host logic: tile-pair planning and the extension-mirror module (CPU only)."""
import numpy as np
import pytest

from ampcor_b200 import plan, synth
from ampcor_b200.ext import ampcor_cuda


def test_uniform_grid_centres():
    # UniformGrid.py:34-54 on 512 x 512 with an 8 x 8 grid: centres 32 + 64 n
    c = plan.uniform_grid((512, 512), (8, 8))
    assert len(c) == 64
    assert c[0] == (32, 32) and c[1] == (32, 96) and c[-1] == (480, 480)
    # uneven split: the leftover border is shared, as m//2 + n t + t//2
    c = plan.uniform_grid((100, 50), (3, 4))
    assert [p[0] for p in c[::4]] == [0 + 16, 33 + 16, 66 + 16]
    assert [p[1] for p in c[:4]] == [1 + 6, 13 + 6, 25 + 6, 37 + 6]


def test_plan_corners_and_validity():
    # Plan.py:160-183: chip corner p - c//2, window corner q - c//2 - pad; invalid pairs dropped
    dom = [(32, 32), (5, 40), (110, 100)]
    cod = plan.constant_codomain(dom, (2, -3))
    ulhc, valid = plan.plan_pairs(dom, cod, (32, 32), (8, 8), (128, 128), (128, 128))
    assert valid.tolist() == [True, False, False]
    assert ulhc.tolist() == [[16, 16, 34 - 16 - 8, 29 - 16 - 8]]


def test_offset_map_product():
    # pkg/ampcor/dom/OffsetMap.py:14-95 (grid-indexed domain/codomain, row-major by default) and
    # Grid.py:34-50 (coarse map from a uniform grid and a constant shift); the refined map moves
    # each valid pair's target point by its offset, dropped pairs stay without a target
    coarse = plan.coarse_map((3, 4), (128, 160), shift=(2, -3))
    assert len(coarse) == 12 and coarse.offset((1, 2)) == 6 and coarse.index(6) == (1, 2)
    assert coarse[(0, 0)] == ((22, 20), (24, 17))
    colmajor = plan.OffsetMap((3, 4), layout=(0, 1))
    assert colmajor.offset((1, 2)) == 7 and colmajor.index(7) == (1, 2)
    ulhc, valid = plan.plan_pairs(coarse.domain, coarse.codomain, (32, 32), (8, 8), (128, 160),
                                  (128, 160))
    offs = np.stack([np.arange(valid.sum()) * 0.25, -np.arange(valid.sum()) * 0.5], 1)
    offs[1] = np.nan  # a pair whose tiles left a raster
    fine = plan.refined_map(coarse, valid, offs)
    field = fine.field()
    assert field.shape == (3, 4, 2)
    k = np.flatnonzero(valid)
    want = np.full((12, 2), np.nan)
    want[k] = np.array([2.0, -3.0]) + offs
    np.testing.assert_array_equal(field.reshape(12, 2), want.astype(np.float32))
    with pytest.raises(IndexError):
        coarse[(3, 0)]


def test_production_grid_is_full():
    w = synth.production_4096()
    assert w.pairs == 14400
    assert w.ulhc[:, 2:].min() >= 0 and w.ulhc[:, 2:].max() + 128 <= 4096


def test_ext_rejects_foreign_worker():
    # ext/ampcor_cuda/sequential.cc:108-126: non-worker capsules raise TypeError
    with pytest.raises(TypeError):
        ampcor_cuda.adjust(object())
    with pytest.raises(TypeError):
        ampcor_cuda.addReference("worker", np.zeros((4, 4), np.complex64), 0, (0, 0), (4, 4))


def test_ext_module_surface():
    for name in ("sequential", "addReference", "addTarget", "adjust", "copyright", "version",
                 "Error"):
        assert hasattr(ampcor_cuda, name)
    assert "ampcor_b200" in ampcor_cuda.version()


class _FakeJob:
    def __init__(self, nbytes):
        self.nbytes = nbytes

    def device_bytes(self):
        return self.nbytes


def test_serving_admission_by_device_memory():
    # jobs are admitted while their bytes fit in what the budget has left, released on
    # completion, and a job larger than the whole budget is refused (it could never run)
    from ampcor_b200.serve import Admission

    a = Admission(100)
    j1, j2, j3, big = _FakeJob(60), _FakeJob(30), _FakeJob(20), _FakeJob(101)
    assert a.try_admit(j1) and a.try_admit(j2)
    assert not a.try_admit(j3) and a.in_use == 90
    assert a.never_fits(big) and not a.never_fits(j3)
    a.release(j1)
    assert a.try_admit(j3) and a.in_use == 50
    a.release(j2)
    a.release(j3)
    assert a.in_use == 0
