"""Batched uneven correlation: many raster pairs of different sizes and tile geometries in one
CUDA-graph launch.

Every distinct geometry (chip, search margin, refinement, zoom) gets one worker, tuned once by
:mod:`ampcor_b200.autotune` (form and refinement chunk); the work of all raster pairs is then
captured into a single CUDA graph on one stream and replayed as one launch.  Each worker's device
memory is sized by a warm-up run before capture, so the captured region allocates nothing.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .serve import grid_corners
from .worker import Worker


@dataclasses.dataclass
class RasterJob:
    ref: "object"            # complex64 device tensor
    tgt: "object"
    ulhc: np.ndarray         # int32 (pairs, 4)
    chip: int
    margin: int
    refine_factor: int = 2
    refine_margin: int = 8
    zoom_factor: int = 8
    field: tuple | None = None   # (constant dy, dx, quadratic amplitude) the generator applied

    @property
    def geometry(self):
        return (self.chip, self.margin, self.refine_factor, self.refine_margin, self.zoom_factor)

    @property
    def pairs(self):
        return int(self.ulhc.shape[0])


def _warp_device(ref, dy0, dx0, quad, seed):
    """Secondary raster: the reference moved by a constant (band-limited Fourier shift) plus a
    smooth quadratic field (bicubic resampling), then complex Gaussian noise at 10 dB."""
    import torch
    import torch.nn.functional as F

    L, S = ref.shape
    dev = ref.device
    ky = torch.fft.fftfreq(L, device=dev, dtype=torch.float64)[:, None]
    kx = torch.fft.fftfreq(S, device=dev, dtype=torch.float64)[None, :]
    shifted = torch.fft.ifft2(torch.fft.fft2(ref.to(torch.complex128)) *
                              torch.exp(-2j * math.pi * (ky * dy0 + kx * dx0))).to(torch.complex64)
    ys = torch.linspace(-1.0, 1.0, L, device=dev)
    xs = torch.linspace(-1.0, 1.0, S, device=dev)
    Y, X = torch.meshgrid(ys, xs, indexing="ij")
    qy = quad * (Y * Y - X * Y * 0.5)
    qx = quad * (X * X + X * Y * 0.5)
    # out(y, x) = in(y - qy, x - qx): sample positions in normalised coordinates
    gy = Y - qy * 2.0 / (L - 1)
    gx = X - qx * 2.0 / (S - 1)
    grid = torch.stack([gx, gy], dim=-1)[None]
    planes = torch.stack([shifted.real, shifted.imag])[None]
    out = F.grid_sample(planes, grid, mode="bicubic", padding_mode="zeros", align_corners=True)[0]
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    nre = torch.randn((L, S), generator=g, device=dev) * math.sqrt(0.05)
    nim = torch.randn((L, S), generator=g, device=dev) * math.sqrt(0.05)
    return torch.complex(out[0] + nre, out[1] + nim).contiguous()


def uneven_jobs(n=16, seed=11, device="cuda:0", shapes=((1024, 1024), (2048, 2048), (4096, 2048),
                                                         (8192, 2048), (2048, 4096)),
                chips=(32, 64, 128), margins=(8, 16, 32, 64), spacing=(16, 128), max_offset=16.0):
    """``n`` seeded raster pairs with uneven shapes and geometries (see module docstring)."""
    import torch

    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(n):
        L, S = shapes[int(rng.integers(len(shapes)))]
        chip = int(rng.choice(chips))
        margin = int(rng.choice(margins))
        sp = int(rng.integers(spacing[0], spacing[1] + 1))
        dy0, dx0 = (float(v) for v in rng.uniform(-0.6, 0.6, 2) * max_offset)
        quad = float(rng.uniform(-0.4, 0.4) * max_offset)
        g = torch.Generator(device=device)
        g.manual_seed(seed * 7919 + k)
        s = 1.0 / math.sqrt(2.0)
        ref = torch.complex(torch.randn((L, S), generator=g, device=device) * s,
                            torch.randn((L, S), generator=g, device=device) * s).contiguous()
        tgt = _warp_device(ref, dy0, dx0, quad, seed * 7919 + k + 1)
        ulhc = grid_corners(L, S, chip, margin, sp)
        jobs.append(RasterJob(ref, tgt, ulhc, chip, margin, field=(dy0, dx0, quad)))
    return jobs


class UnevenBatch:
    """All jobs of a batch captured into one CUDA graph (one worker per geometry)."""

    def __init__(self, jobs, device=0, tune=True, plain=False):
        import torch

        self.jobs = jobs
        self.device = torch.device("cuda", device)
        self.stream = torch.cuda.Stream(device=self.device)
        self.workers = {}
        self.tuning = {}
        self.ulhc = [torch.from_numpy(j.ulhc).to(self.device) for j in jobs]
        self.offsets = [torch.empty((j.pairs, 2), dtype=torch.float32, device=self.device)
                        for j in jobs]
        for j, u in zip(jobs, self.ulhc):
            if j.geometry in self.workers:
                continue
            c, m, f, rm, z = j.geometry
            w = Worker(pairs=max(j.pairs, 1), chip=(c, c), window=(c + 2 * m, c + 2 * m),
                       refine_factor=f, refine_margin=rm, zoom_factor=z, device=device,
                       plain=plain)
            if tune:
                from .autotune import tune as run_tune

                forms = ("plain",) if plain else ("spectral", "tensor", "plain")
                self.tuning[j.geometry] = run_tune(w, j.ref, j.tgt, u, forms=forms,
                                                   chunks=(296, 592, 1184), reps=1,
                                                   use_cache=False)
            self.workers[j.geometry] = w
        self.graph = None

    def _enqueue(self):
        for j, u, out in zip(self.jobs, self.ulhc, self.offsets):
            self.workers[j.geometry].correlate(j.ref, j.tgt, u, offsets=out, stream=self.stream,
                                              synchronize=False)

    def capture(self):
        """Size every worker with one eager run, then record the whole batch as one graph."""
        import torch

        with torch.cuda.stream(self.stream):
            self._enqueue()
        self.stream.synchronize()
        self.check()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=self.stream):
            self._enqueue()
        return self.graph

    def replay(self):
        """Launch the whole batch (one graph launch) on the batch's stream."""
        import torch

        with torch.cuda.stream(self.stream):
            self.graph.replay()

    def check(self):
        for w in self.workers.values():
            w._lib.ampcor_synchronize(w.handle, None)

    @property
    def pairs(self):
        return sum(j.pairs for j in self.jobs)

    def close(self):
        self.graph = None
        for w in self.workers.values():
            w.close()
