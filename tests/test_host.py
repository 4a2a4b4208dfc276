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
