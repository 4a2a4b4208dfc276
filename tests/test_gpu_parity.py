"""Parity of the CUDA path with the oracle (needs a B200).

Every pair of every batch is checked by ``oracle.parity.compare`` (the rules are in its
docstring): integer and sub-pixel cells equal to the FP64 oracle's, offsets then equal bit for
bit, unless the pair's own measured surface error explains a different cell (a near-tie, counted);
peak correlation within 1e-5 relative; every coarse and refined surface within 2e-5 absolute.
The production configuration (14,400 pairs) and its heavy-tailed variant are checked in full.
"""
import numpy as np
import pytest

import oracle
from oracle import parity
from ampcor_b200 import synth
from ampcor_b200.worker import DIAG_DTYPE, Error, Worker
from ampcor_b200.ext import ampcor_cuda

from fixtures import placement_identity

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SURF_ATOL = parity.SURF_ATOL

FORMS = ["spectral", "tensor", "plain"]


def run_device(w: synth.Workload, ulhc=None, surfaces=True, form="tensor", deramp=False):
    ulhc = w.ulhc if ulhc is None else ulhc
    worker = Worker(pairs=len(ulhc), chip=(w.chip, w.chip), window=(w.window, w.window),
                    refine_factor=w.refine_factor, refine_margin=w.refine_margin,
                    zoom_factor=w.zoom_factor, plain=(form == "plain"), deramp=deramp)
    if worker.form != form:
        worker.configure(form)
    assert worker.form == form
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


_ORACLE = {}


def oracle_of(w, ulhc=None, deramp=False, key=None):
    """The oracle's run of a batch (cached per workload when ``key`` is given)."""
    ulhc = w.ulhc if ulhc is None else ulhc
    if key is not None and (key, deramp) in _ORACLE:
        return _ORACLE[(key, deramp)]
    orc = parity.oracle_run(w.ref, w.tgt, ulhc, w.chip, w.window, w.refine_factor,
                            w.refine_margin, w.zoom_factor, deramp=deramp)
    if key is not None:
        _ORACLE[(key, deramp)] = orc
    return orc


def check_parity(w, ulhc, gpu, label, deramp=False, orc=None):
    orc = orc if orc is not None else oracle_of(w, ulhc, deramp)
    rep = parity.compare(orc, gpu["offsets"], gpu["diag"], gpu["coarse"], gpu["refined"])
    assert not rep["failures"], f"{label}: {parity.summary(rep)}"
    assert rep["max_abs_err_non_excused_px"] == 0.0, label
    print(f"{label}: {parity.summary(rep)}")
    return rep


@pytest.mark.parametrize("form", FORMS)
def test_deramp_parity(form):
    # speckle off baseband (a Doppler ramp): with the opt-in deramp every form matches the FP64
    # oracle's deramped pipeline and lands on the zoom grid's rounding of the applied shift
    w = synth.doppler_512()
    gpu = run_device(w, form=form, deramp=True)
    check_parity(w, w.ulhc, gpu, f"doppler_512 deramp {form}", deramp=True,
                 orc=oracle_of(w, deramp=True, key="doppler_512"))
    assert np.abs(gpu["offsets"] - w.truth).max() <= 1.0 / 16 + 1e-6


@pytest.mark.parametrize("form", FORMS)
def test_plain_512_parity(form):
    w = synth.plain_512()
    gpu = run_device(w, form=form)
    rep = check_parity(w, w.ulhc, gpu, "plain_512", orc=oracle_of(w, key="plain_512"))
    assert rep["pairs_excused"] == 0
    assert np.all(gpu["offsets"] == np.float32([3.375, -2.75]))


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("dc", [30.0, 300.0])
def test_large_dc_offset_parity(form, dc):
    # a strong steady return under the speckle (amplitudes near dc, variations of order 1): the
    # window variances S2 - S1^2 / R^2 cancel in proportion to dc^2, the stress the FP64 box
    # statistics and the centred in-kernel column sums are there for
    base = synth.plain_512()
    w = synth.Workload(f"plain_512_dc{int(dc)}", (base.ref + np.complex64(dc)).astype(np.complex64),
                       (base.tgt + np.complex64(dc)).astype(np.complex64), base.ulhc, base.centres,
                       32, 8, 2, 4, 4, base.truth)
    gpu = run_device(w, form=form)
    rep = check_parity(w, w.ulhc, gpu, f"plain_512 + {dc} {form}", orc=oracle_of(w, key=w.name))
    assert rep["pairs_checked"] == 64


@pytest.mark.parametrize("form", FORMS)
def test_golden_plain_512_on_gpu(form):
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "plain_512.npz"))
    gpu = run_device(synth.plain_512(), form=form, surfaces=False)
    assert np.array_equal(gpu["offsets"], g["offsets"])
    assert np.array_equal(gpu["diag"]["coarse_u"], g["coarse_cpu_argmax"][:, 0])
    assert np.array_equal(gpu["diag"]["coarse_v"], g["coarse_cpu_argmax"][:, 1])


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("R,M", [(32, 8), (64, 32)])
def test_placement_identity(R, M, form):
    # correlate.cc:279-303 (gamma = 1 at the placement, 10 eps_f in FP32 there; FP32 sums of
    # R^2 terms here, so 1e-5), maxcor.cc:296-312 (argmax = placement), nudge.cc:204-225
    ref, tgt, ulhc = placement_identity(R, M, seed=5)
    W, C = R + 2 * M, 2 * M + 1
    w = synth.Workload("identity", ref, tgt, ulhc, np.zeros((len(ulhc), 2)), R, M, 2,
                       min(4, M), 4, None)
    gpu = run_device(w, surfaces=True, form=form)
    d = gpu["diag"]
    i, j = np.divmod(np.arange(C * C), C)
    assert np.array_equal(d["coarse_u"], i) and np.array_equal(d["coarse_v"], j)
    np.testing.assert_allclose(gpu["coarse"][np.arange(C * C), i, j], 1.0, atol=1e-5)
    E = R + 2 * w.refine_margin
    assert d["top"].min() >= 0 and d["top"].max() <= W - E
    assert d["left"].min() >= 0 and d["left"].max() <= W - E


def _subset(w, n, seed=0):
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(w.pairs, size=n, replace=False))
    return idx


@pytest.mark.parametrize("form", FORMS)
def test_production_full_job_parity(form):
    # all 14,400 pairs of the benchmark job against the FP64 oracle, pair by pair
    w = synth.production_4096()
    gpu = run_device(w, form=form)
    rep = check_parity(w, w.ulhc, gpu, f"production_4096 {form}", orc=oracle_of(w, key="production_4096"))
    assert rep["pairs_checked"] == 14400
    assert rep["pairs_excused"] <= 144, parity.summary(rep)  # at most 1 % near-ties


@pytest.mark.parametrize("form", FORMS)
def test_heavy_tail_full_job_parity(form):
    # the precision configuration: Rayleigh speckle with 1 % bright scatterers at +30 dB
    w = synth.production_4096(heavy_tail=True)
    gpu = run_device(w, form=form)
    rep = check_parity(w, w.ulhc, gpu, f"heavy_tail_4096 {form}",
                       orc=oracle_of(w, key="heavy_tail_4096"))
    assert rep["pairs_checked"] == 14400
    assert rep["pairs_excused"] <= 144, parity.summary(rep)  # at most 1 % near-ties


@pytest.mark.parametrize("form", FORMS)
def test_production_full_size_properties(form):
    # all 14,400 pairs: finite, near the applied field, and each result identical whether the
    # pair runs in the full batch or in a small one (no cross-pair dependence)
    w = synth.production_4096()
    full = run_device(w, form=form, surfaces=False)
    assert np.isfinite(full["offsets"]).all()
    err = np.abs(full["offsets"] - w.truth)
    assert np.quantile(err, 0.99) < 0.2
    idx = _subset(w, 300, seed=2)
    part = run_device(w, ulhc=w.ulhc[idx], form=form, surfaces=False)
    assert np.array_equal(part["offsets"], full["offsets"][idx])
    assert np.array_equal(part["diag"], full["diag"][idx])
    again = run_device(w, form=form, surfaces=False)
    assert np.array_equal(again["offsets"], full["offsets"])


def test_host_path_matches_device_path():
    w = synth.plain_512()
    worker = Worker(pairs=w.pairs, chip=(32, 32), window=(48, 48), refine_factor=2,
                    refine_margin=4, zoom_factor=4)
    off, diag = worker.correlate(w.ref, w.tgt, w.ulhc, diag=True)
    dev = run_device(w, form=worker.form, surfaces=False)
    assert np.array_equal(off, dev["offsets"])
    assert np.array_equal(diag, dev["diag"])


@pytest.mark.parametrize("order", ["reversed", "shuffled"])
def test_host_path_bands_any_pair_order(order):
    # host-buffer jobs upload the rasters in bands and correlate the pairs whose tiles are up;
    # pairs out of raster order only delay the bands, the offsets stay those of the device path
    w = synth.plain_512()
    perm = np.arange(w.pairs)[::-1] if order == "reversed" else np.random.default_rng(5).permutation(w.pairs)
    ulhc = np.ascontiguousarray(w.ulhc[perm])
    worker = Worker(pairs=w.pairs, chip=(32, 32), window=(48, 48), refine_factor=2,
                    refine_margin=4, zoom_factor=4)
    off, diag = worker.correlate(w.ref, w.tgt, ulhc, diag=True)
    dev = run_device(w, form=worker.form, surfaces=False)
    assert np.array_equal(off, dev["offsets"][perm])
    assert np.array_equal(diag, dev["diag"][perm])


def test_extension_mirror_matches_raster_path():
    # the reference's call sequence (pkg/ampcor/correlators/CUDA.py:45-58)
    w = synth.plain_512()
    worker = ampcor_cuda.sequential(w.pairs, (32, 32), (48, 48), 4, 2, 4)
    for idx, (rl, rs, tl, ts) in enumerate(w.ulhc):
        ampcor_cuda.addReference(worker, w.ref, idx, (rl, rs), (rl + 32, rs + 32))
        ampcor_cuda.addTarget(worker, w.tgt, idx, (tl, ts), (tl + 48, ts + 48))
    offsets = ampcor_cuda.adjust(worker)
    assert isinstance(offsets, tuple) and len(offsets) == w.pairs
    assert all(isinstance(o, tuple) and len(o) == 2 for o in offsets)
    dev = run_device(w, form=ampcor_cuda._worker(worker).form, surfaces=False)
    assert np.array_equal(np.array(offsets, np.float32), dev["offsets"])


def test_ref_compat_flag():
    w = synth.plain_512()
    worker = Worker(pairs=w.pairs, chip=(32, 32), window=(48, 48), refine_factor=2,
                    refine_margin=4, zoom_factor=4, ref_compat=True)
    off = worker.correlate(w.ref, w.tgt, w.ulhc)
    oc, _ = oracle.adjust(w.ref, w.tgt, w.ulhc, 32, 48, 2, 4, 4, ref_compat=True)
    assert np.array_equal(off, oc)


def test_out_of_bounds_pair_reports_and_is_nan():
    w = synth.plain_512()
    ulhc = w.ulhc[:4].copy()
    ulhc[2, 2] = 500   # window leaves the 512-line raster
    worker = Worker(pairs=4, chip=(32, 32), window=(48, 48), refine_factor=2, refine_margin=4,
                    zoom_factor=4)
    dev = torch.device("cuda:0")
    with pytest.raises(Error) as e:
        worker.correlate(torch.from_numpy(w.ref).to(dev), torch.from_numpy(w.tgt).to(dev),
                         torch.from_numpy(ulhc).to(dev))
    assert "leave their raster" in str(e.value)
    off = worker.correlate(torch.from_numpy(w.ref).to(dev), torch.from_numpy(w.tgt).to(dev),
                           torch.from_numpy(ulhc).to(dev), synchronize=False)
    torch.cuda.synchronize()
    o = off.cpu().numpy()
    assert np.isnan(o[2]).all() and np.isfinite(o[[0, 1, 3]]).all()


@pytest.mark.parametrize("form", ["tensor", "spectral"])
def test_forms_agree_with_plain(form):
    # a form and the plain form on the same pairs: same integer and sub-pixel cells except
    # near-ties, surfaces within the parity tolerance of each other
    w = synth.production_4096()
    idx = _subset(w, 256, seed=3)
    t = run_device(w, ulhc=w.ulhc[idx], surfaces=True, form=form)
    p = run_device(w, ulhc=w.ulhc[idx], surfaces=True, form="plain")
    np.testing.assert_allclose(t["coarse"], p["coarse"], atol=SURF_ATOL, rtol=0)
    np.testing.assert_allclose(t["refined"], p["refined"], atol=SURF_ATOL, rtol=0)
    assert (t["offsets"] == p["offsets"]).all(axis=1).mean() > 0.98


@pytest.mark.parametrize("shape,chip", [((500, 514), 32), ((590, 601), 32)])
def test_copy_engine_edge_cases_parity(shape, chip):
    """The staged kernels take their windows through the copy engine, which wants raster lines of
    whole 16-byte units.  Lines of 514 samples (the amplitude raster's lines are not 16-byte
    multiples, the complex raster's are: the coarse stage falls back to spec_kernel, the window
    refinement stays staged) and of 601 samples (neither: both fall back) still give every pair
    the FP64 oracle's offsets.  (Refined tiles are always whole 16-byte rows: tiles are multiples
    of 8 samples.)"""
    ref = synth.speckle(shape, 3)
    tgt = (synth.fourier_shift(ref, 2.3, -1.6) + synth.noise(shape, 10.0, 4)).astype(np.complex64)
    centres = synth.uniform_grid(shape, (6, 6))
    ulhc, kept = synth._grid_pairs(shape, centres, chip, 8)
    w = synth.Workload("edges", ref, tgt, ulhc, kept, chip, 8, 2, 4, 4, None)
    gpu = run_device(w, form="spectral")
    check_parity(w, w.ulhc, gpu, f"{shape} chip {chip}")
