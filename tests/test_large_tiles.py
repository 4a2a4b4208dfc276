"""Tile geometries beyond one CTA's shared memory (needs a B200): the reference's own default
chip of 128 x 128 with a 32 px padding (pkg/ampcor/correlators/MGA.py:28-42, the geometry of its
stage tests, tests/libampcor_cuda/correlate.cc:60-71) and search margins of 64 px.

Windows too large for one FFT tile are correlated in chip blocks (spec_block_kernel, one tile per
block, reduced per pair by spec_reduce_kernel); refined tiles of 128 and 144 samples are
upsampled through a per-pair buffer (spec_refine_big_kernel).  Only the spectral form covers these
geometries.  Every pair is checked against the FP64 oracle by oracle.parity.compare.
"""
import numpy as np
import pytest

from oracle import parity
from ampcor_b200 import synth
from ampcor_b200.worker import DIAG_DTYPE, Error, Worker

from fixtures import placement_identity

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def run(w, ulhc=None, surfaces=True):
    ulhc = w.ulhc if ulhc is None else ulhc
    worker = Worker(pairs=len(ulhc), chip=(w.chip, w.chip), window=(w.window, w.window),
                    refine_factor=w.refine_factor, refine_margin=w.refine_margin,
                    zoom_factor=w.zoom_factor)
    assert worker.form == "spectral"
    dev = torch.device("cuda:0")
    ref = torch.from_numpy(w.ref).to(dev)
    tgt = torch.from_numpy(w.tgt).to(dev)
    u = torch.from_numpy(np.ascontiguousarray(ulhc)).to(dev)
    P = len(ulhc)
    diag = torch.zeros((P, DIAG_DTYPE.itemsize), dtype=torch.uint8, device=dev)
    cs = rs = None
    if surfaces:
        cs = torch.zeros((P, worker.coarse_dim, worker.coarse_dim), dtype=torch.float32, device=dev)
        rs = torch.zeros((P, worker.refined_dim, worker.refined_dim), dtype=torch.float32, device=dev)
    off = worker.correlate(ref, tgt, u, diag=diag, coarse_surfaces=cs, refined_surfaces=rs)
    out = dict(offsets=off.cpu().numpy(), diag=diag.cpu().numpy().view(DIAG_DTYPE).reshape(P))
    if surfaces:
        out["coarse"] = cs.cpu().numpy()
        out["refined"] = rs.cpu().numpy()
    worker.close()
    return out


def check(w, gpu, ulhc=None):
    ulhc = w.ulhc if ulhc is None else ulhc
    orc = parity.oracle_run(w.ref, w.tgt, ulhc, w.chip, w.window, w.refine_factor,
                            w.refine_margin, w.zoom_factor)
    rep = parity.compare(orc, gpu["offsets"], gpu["diag"], gpu["coarse"], gpu["refined"])
    print(f"{w.name}: {parity.summary(rep)}")
    assert not rep["failures"], parity.summary(rep)
    assert rep["max_abs_err_non_excused_px"] == 0.0
    assert rep["pairs_excused"] <= max(2, len(ulhc) // 100), parity.summary(rep)
    return rep


@pytest.mark.parametrize("R,M,step", [(128, 32, 1), (64, 64, 4), (32, 64, 4), (128, 64, 8)])
def test_placement_identity_large(R, M, step):
    # correlate.cc:279-303 (gamma = 1 at the placement), maxcor.cc:296-312 (argmax = placement),
    # nudge.cc:204-225 (the refinement neighbourhood stays inside the window)
    fx = placement_identity(R, M, seed=5, step=step)
    ref, tgt, ulhc = fx[:3]
    W, C = R + 2 * M, 2 * M + 1
    cells = fx[3] if step > 1 else np.stack(np.divmod(np.arange(C * C), C), axis=1)
    w = synth.Workload("identity", ref, tgt, ulhc, np.zeros((len(ulhc), 2)), R, M, 2, 8, 4, None)
    gpu = run(w)
    d = gpu["diag"]
    assert np.array_equal(d["coarse_u"], cells[:, 0]) and np.array_equal(d["coarse_v"], cells[:, 1])
    P = len(ulhc)
    np.testing.assert_allclose(gpu["coarse"][np.arange(P), cells[:, 0], cells[:, 1]], 1.0, atol=1e-5)
    E = R + 2 * w.refine_margin
    assert d["top"].min() >= 0 and d["top"].max() <= W - E
    assert d["left"].min() >= 0 and d["left"].max() <= W - E


def test_reference_default_geometry_full_job_parity():
    # 3,600 pairs of 128 x 128 chips, +-32 px, refine 2 / 8, zoom 8, on the production rasters
    w = synth.reference_default_4096()
    gpu = run(w)
    rep = check(w, gpu)
    assert rep["pairs_checked"] == 3600
    err = np.abs(gpu["offsets"] - w.truth)
    assert np.quantile(err, 0.99) < 0.2


@pytest.mark.parametrize("chip,margin,n,spacing", [(64, 64, 10, 300), (128, 64, 8, 400),
                                                   (32, 64, 10, 300), (128, 16, 8, 400)])
def test_large_margin_parity(chip, margin, n, spacing):
    w = synth.grid_4096(chip, margin, n, spacing)
    check(w, run(w))


def test_arena_path_at_chip_128():
    # the pair-by-pair arena (the reference's addReferenceTile / addTargetTile / adjust): its
    # windows are not a raster, so the placement statistics come from the window itself
    # (spec_tile_stats_kernel); offsets equal to the raster path's
    w = synth.reference_default_4096()
    idx = np.linspace(0, w.pairs - 1, 24).round().astype(int)
    worker = Worker(pairs=len(idx), chip=(128, 128), window=(192, 192), refine_factor=2,
                    refine_margin=8, zoom_factor=8)
    for k, p in enumerate(idx):
        c, win = w.arena_tiles(p)
        worker.add_reference(k, np.ascontiguousarray(c))
        worker.add_target(k, np.ascontiguousarray(win))
    off = worker.adjust()
    worker.close()
    raster = run(w, ulhc=w.ulhc[idx], surfaces=False)
    assert np.array_equal(off, raster["offsets"])


def test_plain_and_tensor_forms_refuse_the_large_geometry():
    w = synth.reference_default_4096()
    worker = Worker(pairs=4, chip=(128, 128), window=(192, 192), refine_factor=2, refine_margin=8,
                    zoom_factor=8)
    for form in ("plain", "tensor"):
        with pytest.raises(Error) as e:
            worker.configure(form)
        assert "AMPCOR_E_SHAPE" in str(e.value)
    assert worker.form == "spectral"
    worker.close()
    with pytest.raises(Error):
        Worker(pairs=4, chip=(128, 128), window=(192, 192), plain=True)
