"""Writes tests/golden/plain_512.npz: the oracle's answer on the CPU-runnable configuration
(512x512 speckle shifted by (+3.4, -2.7) px, 8x8 pairs of 32x32 chips, +-8 px, refine 2/4,
zoom 4).  Re-run only when the oracle's definition changes on purpose:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from ampcor_b200 import synth  # noqa: E402

w = synth.plain_512()
off, diag = oracle.adjust(w.ref, w.tgt, w.ulhc, 32, 48, 2, 4, 4)
arg, gap = oracle.coarse_cpu(w.ref, w.tgt, w.ulhc, 32, 48)
np.savez_compressed(
    os.path.join(os.path.dirname(os.path.abspath(__file__)), "plain_512.npz"),
    ulhc=w.ulhc, offsets=off, coarse_cpu_argmax=arg, coarse_cpu_gap=gap,
    coarse_u=diag["coarse_u"], coarse_v=diag["coarse_v"], fine_p=diag["fine_p"],
    fine_q=diag["fine_q"], refined_peak=diag["refined_peak"], coarse_peak=diag["coarse_peak"],
    zoom_gap=diag["zoom_gap"],
)
print("wrote plain_512.npz")
