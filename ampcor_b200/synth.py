"""Seeded synthetic raster pairs for the correlator workloads.

The reference measures on a real ALOS-style SLC pair that is not distributed with it; these
generators stand in for it with the statistics of single-look SAR data:

* speckle: circular complex Gaussian pixels of unit variance (amplitude Rayleigh);
* the secondary raster is the reference moved by a known offset field (a Fourier-domain
  sub-pixel shift, or a smooth quadratic field applied with FP64 windowed-sinc resampling) plus
  complex Gaussian noise at the requested SNR.

``workload(name)`` returns a :class:`Workload` with the rasters, the tile-pair corners and the
correlator geometry of a named benchmark configuration.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np

from .plan import constant_codomain, plan_pairs, uniform_grid

HERE = os.path.dirname(os.path.abspath(__file__))
# generated rasters are cached per machine, outside the source tree
CACHE = os.environ.get("AMPCOR_SYNTH_CACHE", os.path.join("/tmp", "ampcor_b200_synth"))


def speckle(shape, seed) -> np.ndarray:
    """Circular complex Gaussian raster with unit variance (complex64)."""
    rng = np.random.default_rng(seed)
    z = np.empty(shape, np.complex64)
    s = np.float32(np.sqrt(0.5))
    z.real = rng.standard_normal(shape, dtype=np.float32) * s
    z.imag = rng.standard_normal(shape, dtype=np.float32) * s
    return z


def noise(shape, snr_db, seed) -> np.ndarray:
    """Complex Gaussian noise whose variance is 10^(-snr/10) of a unit-variance signal."""
    var = 10.0 ** (-snr_db / 10.0)
    return (speckle(shape, seed) * np.float32(np.sqrt(var))).astype(np.complex64)


def fourier_shift(x, dy, dx) -> np.ndarray:
    """x moved by (dy, dx) pixels: out(y, x) = in(y - dy, x - dx), by an FP64 phase ramp."""
    X = np.fft.fft2(x.astype(np.complex128))
    ky = np.fft.fftfreq(x.shape[0])[:, None]
    kx = np.fft.fftfreq(x.shape[1])[None, :]
    X *= np.exp(-2j * np.pi * (ky * dy + kx * dx))
    return np.fft.ifft2(X).astype(np.complex64)


def quadratic_field(seed, max_px):
    """Coefficients (cy, cx) of a bivariate quadratic offset field with |offset| <= max_px.

    dy = cy . (1, Y, X, Y^2, XY, X^2) in normalised coordinates X, Y in [-1, 1].
    """
    rng = np.random.default_rng(seed)
    cy = rng.uniform(-1.0, 1.0, 6)
    cx = rng.uniform(-1.0, 1.0, 6)
    g = np.linspace(-1.0, 1.0, 201)
    Y, X = np.meshgrid(g, g, indexing="ij")
    basis = np.stack([np.ones_like(X), Y, X, Y * Y, X * Y, X * X])
    mag = np.sqrt(np.tensordot(cy, basis, 1) ** 2 + np.tensordot(cx, basis, 1) ** 2).max()
    scale = max_px / mag
    return cy * scale, cx * scale


def field_at(coefs, shape, y, x):
    """Evaluate a quadratic field at pixel coordinates."""
    H, W = shape
    Y = (np.asarray(y, np.float64) - H / 2.0) / (H / 2.0)
    X = (np.asarray(x, np.float64) - W / 2.0) / (W / 2.0)
    b = np.stack([np.ones_like(X), Y, X, Y * Y, X * Y, X * X])
    return np.tensordot(coefs, b, 1)


_synth_lib = None


def _warp_lib():
    global _synth_lib
    if _synth_lib is None:
        path = os.path.join(HERE, "libampcor_synth.so")
        if not os.path.exists(path):
            from .build import build

            build()
        lib = ctypes.CDLL(path)
        lib.synth_warp.restype = None
        lib.synth_warp.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong,
                                   ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p]
        _synth_lib = lib
    return _synth_lib


def warp(x, cy, cx) -> np.ndarray:
    """out(y, x) = in(y - dy, x - dx) with a quadratic (dy, dx), FP64 windowed sinc."""
    x = np.ascontiguousarray(x, np.complex64)
    out = np.empty_like(x)
    cy = np.ascontiguousarray(cy, np.float64)
    cx = np.ascontiguousarray(cx, np.float64)
    _warp_lib().synth_warp(x.ctypes.data, out.ctypes.data, x.shape[0], x.shape[1],
                           cy.ctypes.data, cx.ctypes.data)
    return out


@dataclasses.dataclass
class Workload:
    name: str
    ref: np.ndarray            # complex64 reference raster
    tgt: np.ndarray            # complex64 secondary raster
    ulhc: np.ndarray           # int32 (pairs, 4): chip line/sample, window line/sample
    centres: np.ndarray        # (pairs, 2) chip centres
    chip: int
    margin: int
    refine_factor: int
    refine_margin: int
    zoom_factor: int
    truth: np.ndarray | None   # (pairs, 2) offsets the generator applied at the chip centres

    @property
    def window(self) -> int:
        return self.chip + 2 * self.margin

    @property
    def pairs(self) -> int:
        return int(self.ulhc.shape[0])

    def arena_tiles(self, pid):
        """(chip, window) complex64 tiles of pair pid, as the reference fills its arena."""
        rl, rs, tl, ts = (int(v) for v in self.ulhc[pid])
        c, w = self.chip, self.window
        return self.ref[rl:rl + c, rs:rs + c], self.tgt[tl:tl + w, ts:ts + w]


def _grid_pairs(ref_shape, centres, chip, margin):
    centres = [tuple(int(v) for v in c) for c in centres]
    ulhc, valid = plan_pairs(centres, constant_codomain(centres), (chip, chip),
                             (margin, margin), ref_shape, ref_shape)
    kept = np.asarray(centres, np.int64)[valid]
    return ulhc, kept


def plain_512():
    """512x512 speckle, secondary Fourier-shifted by (+3.4, -2.7) px plus noise at 10 dB;
    8x8 UniformGrid of 32x32 chips, +-8 px search, refine 2 / margin 4, zoom 4."""
    ref = speckle((512, 512), 0)
    tgt = (fourier_shift(ref, 3.4, -2.7) + noise((512, 512), 10.0, 1)).astype(np.complex64)
    centres = uniform_grid((512, 512), (8, 8))
    ulhc, kept = _grid_pairs(ref.shape, centres, 32, 8)
    truth = np.tile(np.array([[3.4, -2.7]]), (len(kept), 1))
    return Workload("plain_512", ref, tgt, ulhc, kept, 32, 8, 2, 4, 4, truth)


def doppler_512(ramp=(0.1, 0.45), band=0.6, shift=(3.4, -2.7)):
    """plain_512's geometry on oversampled speckle whose spectrum sits off baseband, as SAR data
    with a Doppler centroid does: band-limited speckle (a fraction ``band`` of each axis'
    spectrum), the secondary Fourier-shifted by ``shift`` px, both multiplied by the phase ramp
    exp(2 pi i (ramp[0] line + ramp[1] sample)) (cycles per sample).  Without a deramp the
    band-limited refinement's zero padding cuts through the shifted spectrum."""
    base = speckle((512, 512), 0).astype(np.complex128)
    B = np.fft.fft2(base)
    fy = np.fft.fftfreq(512)[:, None]
    fx = np.fft.fftfreq(512)[None, :]
    B[(np.abs(fy) > band / 2) | (np.abs(fx) > band / 2)] = 0.0
    base = np.fft.ifft2(B)
    base /= np.sqrt((np.abs(base) ** 2).mean())
    y, x = np.mgrid[0:512, 0:512]
    ph = np.exp(2j * np.pi * (ramp[0] * y + ramp[1] * x))
    ref = (ph * base).astype(np.complex64)
    tgt = (ph * fourier_shift(base.astype(np.complex64), *shift)).astype(np.complex64)
    centres = uniform_grid((512, 512), (8, 8))
    ulhc, kept = _grid_pairs(ref.shape, centres, 32, 8)
    truth = np.tile(np.array([list(shift)]), (len(kept), 1))
    return Workload("doppler_512", ref, tgt, ulhc, kept, 32, 8, 2, 4, 4, truth)


def _cached(key, make):
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, key + ".npy")
    if os.path.exists(path):
        try:
            return np.load(path, mmap_mode=None)
        except Exception:
            pass
    arr = make()
    tmp = os.path.join(CACHE, f"{key}.{os.getpid()}.tmp.npy")
    np.save(tmp, arr)
    os.replace(tmp, path)
    return arr


def production_4096(n=120, heavy_tail=False):
    """4096x4096 speckle, secondary warped by a seeded quadratic field (|offset| <= 10 px) plus
    noise at 10 dB; n x n chips of 64x64 on centres 64 + 33 k, +-32 px search, refine 2 /
    margin 8, zoom 8.  With heavy_tail, 1% of the reference pixels are bright point scatterers
    (+30 dB) before the warp."""
    shape = (4096, 4096)
    cy, cx = quadratic_field(3, 10.0)
    tag = "ht" if heavy_tail else "sp"

    def make_ref():
        r = speckle(shape, 1)
        if heavy_tail:
            rng = np.random.default_rng(4)
            mask = rng.random(shape) < 0.01
            r[mask] *= np.float32(10.0 ** (30.0 / 20.0))
        return r

    ref = _cached(f"prod4096_{tag}_ref", make_ref)

    def make_tgt():
        return (warp(ref, cy, cx) + noise(shape, 10.0, 2)).astype(np.complex64)

    tgt = _cached(f"prod4096_{tag}_tgt", make_tgt)
    ticks = [64 + 33 * k for k in range(n)]
    centres = [(a, b) for a in ticks for b in ticks]
    ulhc, kept = _grid_pairs(shape, centres, 64, 32)
    truth = np.stack([field_at(cy, shape, kept[:, 0], kept[:, 1]),
                      field_at(cx, shape, kept[:, 0], kept[:, 1])], axis=1)
    name = "heavy_tail_4096" if heavy_tail else "production_4096"
    return Workload(name, ref, tgt, ulhc, kept, 64, 32, 2, 8, 8, truth)


def grid_4096(chip, margin, n, spacing, heavy_tail=False, refine_margin=8, zoom=8):
    """production_4096's rasters with another tile geometry: an n x n grid of chip x chip tiles
    spaced ``spacing`` px apart, centred on the raster, +-margin px search, refine 2 / margin
    ``refine_margin``, zoom ``zoom``.  Pairs whose window would leave the raster are dropped as
    Plan.assemble drops them."""
    base = production_4096(heavy_tail=heavy_tail)
    shape = base.ref.shape
    cy, cx = quadratic_field(3, 10.0)
    span = spacing * (n - 1)
    first = (shape[0] - span) // 2
    ticks = [first + spacing * k for k in range(n)]
    centres = [(a, b) for a in ticks for b in ticks]
    ulhc, kept = _grid_pairs(shape, centres, chip, margin)
    truth = np.stack([field_at(cy, shape, kept[:, 0], kept[:, 1]),
                      field_at(cx, shape, kept[:, 0], kept[:, 1])], axis=1)
    name = f"chip{chip}_margin{margin}_4096"
    return Workload(name, base.ref, base.tgt, ulhc, kept, chip, margin, 2, refine_margin, zoom, truth)


def reference_default_4096():
    """The reference's default correlation geometry (pkg/ampcor/correlators/MGA.py:28-42:
    128 x 128 chips, 32 px padding, refine factor 2 with an 8 px margin, zoom 8) on
    production_4096's rasters: a 60 x 60 grid of chips 64 px apart, 3,600 pairs."""
    return grid_4096(128, 32, 60, 64)


WORKLOADS = {
    "plain_512": plain_512,
    "production_4096": production_4096,
    "heavy_tail_4096": lambda: production_4096(heavy_tail=True),
    "reference_default_4096": reference_default_4096,
}


def workload(name: str) -> Workload:
    return WORKLOADS[name]()
