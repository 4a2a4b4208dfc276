"""Continuous-batching request loop for correlation jobs.

A job is a raster pair plus its tile-pair corners and geometry (chip, search margin, refinement,
zoom).  Jobs arrive over time (a seeded Poisson stream in :func:`poisson_jobs`); the server admits
an arrived job as soon as an execution slot is free and the job fits in the device-memory budget,
so jobs that arrive while others run are started at once and their kernels overlap on the GPU
(every slot has its own CUDA stream and its own workers - a worker's scratch is never shared by
two jobs in flight).  The rasters, corners, offsets and all intermediate surfaces stay in device
memory; only the request (pinned host rasters) and the offsets cross PCIe.  Latency is measured
from a job's arrival to the completion event of its offsets.

Results do not depend on what else runs: each pair's computation is fixed-order and independent of
the other pairs and jobs, which ``tests/test_serving.py`` checks (alone vs in the mix).
"""
from __future__ import annotations

import dataclasses
import math
import time
from collections import deque

import numpy as np

from .worker import Worker


@dataclasses.dataclass
class Job:
    jid: int
    arrival: float                 # seconds after the stream starts
    ref: "object"                  # complex64 raster (pinned host or device tensor)
    tgt: "object"
    ulhc: np.ndarray               # int32 (pairs, 4)
    chip: int
    margin: int
    refine_factor: int
    refine_margin: int
    zoom_factor: int
    truth: tuple | None = None     # applied (dy, dx), when known
    # filled by the server
    start: float | None = None
    done: float | None = None
    offsets: np.ndarray | None = None
    error: str | None = None       # why the job was refused, if it was

    @property
    def pairs(self):
        return int(self.ulhc.shape[0])

    @property
    def geometry(self):
        return (self.chip, self.margin, self.refine_factor, self.refine_margin, self.zoom_factor)

    def device_bytes(self):
        """Device memory the job holds while it runs: both rasters (complex64), its corners and
        its offsets.  The workers' own scratch (sized once per geometry and slot by
        :meth:`Server.warm`) is outside the budget the server admits against."""
        return (self.ref.numel() + self.tgt.numel()) * 8 + self.pairs * (16 + 8)


class Admission:
    """First-come admission of jobs by device memory.  A job is admitted when its bytes fit in
    what the budget has left; the oldest waiting job blocks the ones behind it (no overtaking),
    and a job larger than the whole budget is refused at once, since it could never run."""

    def __init__(self, budget):
        self.budget = int(budget)
        self.in_use = 0

    def never_fits(self, job):
        return job.device_bytes() > self.budget

    def try_admit(self, job):
        need = job.device_bytes()
        if self.in_use + need > self.budget:
            return False
        self.in_use += need
        return True

    def release(self, job):
        self.in_use -= job.device_bytes()


def synth_pair(lines, samples, shift, seed, device, snr_db=10.0):
    """Seeded speckle raster pair on the device: the secondary is the reference moved by the
    sub-pixel ``shift`` (phase ramp in the Fourier domain) plus complex Gaussian noise."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    s = 1.0 / math.sqrt(2.0)
    re = torch.randn((lines, samples), generator=g, device=device, dtype=torch.float32) * s
    im = torch.randn((lines, samples), generator=g, device=device, dtype=torch.float32) * s
    ref = torch.complex(re, im)
    ky = torch.fft.fftfreq(lines, device=device, dtype=torch.float64)[:, None]
    kx = torch.fft.fftfreq(samples, device=device, dtype=torch.float64)[None, :]
    ramp = torch.exp(-2j * math.pi * (ky * shift[0] + kx * shift[1]))
    tgt = torch.fft.ifft2(torch.fft.fft2(ref.to(torch.complex128)) * ramp).to(torch.complex64)
    nvar = 10.0 ** (-snr_db / 10.0)
    nre = torch.randn((lines, samples), generator=g, device=device, dtype=torch.float32)
    nim = torch.randn((lines, samples), generator=g, device=device, dtype=torch.float32)
    tgt = tgt + torch.complex(nre, nim) * float(math.sqrt(nvar / 2.0))
    return ref.contiguous(), tgt.contiguous()


def grid_corners(lines, samples, chip, margin, spacing):
    """Chip/window corners of a regular grid of tile centres, all inside the rasters."""
    half = chip // 2 + margin
    ys = np.arange(half, lines - half - chip % 2 + 1, spacing)
    xs = np.arange(half, samples - half - chip % 2 + 1, spacing)
    cy, cx = np.meshgrid(ys, xs, indexing="ij")
    cy, cx = cy.ravel(), cx.ravel()
    ulhc = np.stack([cy - chip // 2, cx - chip // 2, cy - chip // 2 - margin, cx - chip // 2 - margin], 1)
    return ulhc.astype(np.int32)


def poisson_jobs(n_jobs, rate=20.0, seed=7, device="cuda:0", sizes=(1024, 2048, 3072, 4096),
                 chips=(32, 64), margins=(16, 32), zooms=(8, 16), refine_factor=2,
                 refine_margin=8, spacing=(64, 128), pinned=True, square=False):
    """A seeded Poisson stream of jobs (mean ``rate`` jobs/s): raster sides drawn from ``sizes``
    (one side for both axes with ``square``), chip / margin / zoom from their lists, grid spacing
    from ``spacing``, a random sub-pixel shift of at most 8 px.  Rasters are generated on the
    device and, with ``pinned``, copied to pinned host memory so that each job's upload is part of
    its latency."""
    import torch

    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for jid in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        lines = int(rng.choice(sizes))
        samples = lines if square else int(rng.choice(sizes))
        chip = int(rng.choice(chips))
        margin = int(rng.choice(margins))
        zoom = int(rng.choice(zooms))
        sp = int(rng.integers(spacing[0], spacing[1] + 1))
        shift = tuple(float(v) for v in rng.uniform(-8.0, 8.0, 2))
        ref, tgt = synth_pair(lines, samples, shift, seed * 100003 + jid, device)
        if pinned:
            ref = ref.cpu().pin_memory()
            tgt = tgt.cpu().pin_memory()
        ulhc = grid_corners(lines, samples, chip, margin, sp)
        jobs.append(Job(jid, t, ref, tgt, ulhc, chip, margin, refine_factor, refine_margin, zoom,
                        truth=shift))
    return jobs


class Server:
    """Runs jobs with up to ``slots`` in flight on ``device``, admitting by free device memory.

    The budget is ``memory_budget`` bytes, or else 80 % of the device memory that is free once
    :meth:`warm` has created the workers (whose scratch is therefore not counted twice)."""

    def __init__(self, device=0, slots=4, memory_budget=None, plain=False):
        import torch

        self.device = torch.device("cuda", device)
        self.slots = slots
        self.plain = plain
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(slots)]
        self.workers = [dict() for _ in range(slots)]
        self.fixed_budget = memory_budget
        self.admission = Admission(memory_budget if memory_budget is not None else self._free_budget())

    def _free_budget(self):
        import torch

        free, _ = torch.cuda.mem_get_info(self.device)
        return int(free * 0.8)

    @property
    def budget(self):
        return self.admission.budget

    def _worker(self, slot, job):
        ws = self.workers[slot]
        key = job.geometry
        if key not in ws:
            c, m, f, rm, z = key
            ws[key] = Worker(pairs=max(job.pairs, 1), chip=(c, c), window=(c + 2 * m, c + 2 * m),
                             refine_factor=f, refine_margin=rm, zoom_factor=z,
                             device=self.device.index, plain=self.plain)
        return ws[key]

    def warm(self, jobs):
        """Create (and exercise once) every worker the jobs will need, outside the timed loop.

        Each worker runs the largest jobs of its geometry (by raster area, raster width and pair
        count), so that the device buffers it sizes on first use (amplitude rasters, box
        statistics, per-pair results) never grow inside the timed loop; growing one frees
        memory, which waits for the whole device."""
        import torch

        largest = {}
        for job in jobs:
            lines, samples = job.ref.shape
            picks = largest.setdefault(job.geometry, {})
            for key, val in (("area", lines * samples), ("width", samples), ("pairs", job.pairs)):
                if key not in picks or val > picks[key][0]:
                    picks[key] = (val, job)
        warm_jobs = []
        for picks in largest.values():
            for _, job in picks.values():
                if all(job is not j for j in warm_jobs):
                    warm_jobs.append(job)
        for job in warm_jobs:
            for slot in range(self.slots):
                w = self._worker(slot, job)
                with torch.cuda.stream(self.streams[slot]):
                    ref = job.ref.to(self.device, non_blocking=True)
                    tgt = job.tgt.to(self.device, non_blocking=True)
                    u = torch.from_numpy(job.ulhc).to(self.device)
                    w.correlate(ref, tgt, u, stream=self.streams[slot])
        torch.cuda.synchronize(self.device)
        if self.fixed_budget is None:
            torch.cuda.empty_cache()
            self.admission = Admission(self._free_budget())

    def _launch(self, slot, job, now):
        import torch

        st = self.streams[slot]
        w = self._worker(slot, job)
        with torch.cuda.stream(st):
            ref = job.ref.to(self.device, non_blocking=True)
            tgt = job.tgt.to(self.device, non_blocking=True)
            u = torch.from_numpy(job.ulhc).to(self.device, non_blocking=True)
            off = torch.empty((job.pairs, 2), dtype=torch.float32, device=self.device)
            w.correlate(ref, tgt, u, offsets=off, stream=st, synchronize=False)
            host = torch.empty((job.pairs, 2), dtype=torch.float32, pin_memory=True)
            host.copy_(off, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(st)
        job.start = now
        return (job, ev, host, (ref, tgt, u, off))

    def run(self, jobs, realtime=True):
        """Serve ``jobs`` (sorted by arrival).  With ``realtime`` the loop follows the arrival
        clock; otherwise every job is considered arrived at time 0 (a saturation run)."""
        import torch

        torch.cuda.set_device(self.device)
        pending = deque()
        queue = deque(sorted(jobs, key=lambda j: j.arrival))
        running = [None] * self.slots
        t0 = time.perf_counter()
        finished = 0
        while finished < len(jobs):
            now = time.perf_counter() - t0
            while queue and (not realtime or queue[0].arrival <= now):
                pending.append(queue.popleft())
            for s in range(self.slots):
                r = running[s]
                if r is not None and r[1].query():
                    job, ev, host, keep = r
                    job.done = time.perf_counter() - t0
                    job.offsets = host.numpy().copy()
                    self.admission.release(job)
                    running[s] = None
                    finished += 1
            while pending and self.admission.never_fits(pending[0]):
                job = pending.popleft()
                job.error = (f"needs {job.device_bytes()} bytes of device memory, more than the "
                             f"server's budget of {self.admission.budget}")
                job.done = now
                finished += 1
            for s in range(self.slots):
                if running[s] is None and pending:
                    if not self.admission.try_admit(pending[0]):
                        break
                    running[s] = self._launch(s, pending.popleft(), now)
            time.sleep(0.0002)
        for s in range(self.slots):
            for w in self.workers[s].values():
                w._lib.ampcor_synchronize(w.handle, None)
        return jobs


def latency_report(jobs):
    """p50 / p99 job latency (ms), pairs/s over the busy span, and offset error vs the shifts,
    over the jobs that ran (refused ones are counted apart)."""
    refused = [j for j in jobs if j.error]
    jobs = [j for j in jobs if not j.error]
    lat = np.array([(j.done - j.arrival) * 1e3 for j in jobs])
    pairs = sum(j.pairs for j in jobs)
    span = max(j.done for j in jobs) - min(j.arrival for j in jobs)
    errs = [np.abs(j.offsets - np.asarray(j.truth)[None, :]).max() for j in jobs if j.truth]
    return {
        "jobs": len(jobs),
        "refused": len(refused),
        "pairs": pairs,
        "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)),
        "max_ms": float(lat.max()),
        "pairs_per_s": pairs / span,
        "max_offset_error_px": float(max(errs)) if errs else None,
    }
