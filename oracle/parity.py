"""Pair-by-pair comparison of a GPU correlation with the FP64 oracle - TEST INFRASTRUCTURE ONLY.

Used by ``tests/`` and by the CPU-baseline leg of ``bench.py`` (which times the oracle over the
benchmark job and then checks the timed job's own offsets with it); the product never imports it.

Every pair is checked.  A pair's integer or sub-pixel cell may differ from the oracle's only when
the difference is explained by the pair's own error bound, and such pairs are counted:

* coarse cell (integer offsets): delta_c = the largest |gamma_gpu - gamma_oracle| over the pair's
  coarse surface (all C^2 placements, the FP32 form's measured error on that pair).  The GPU cell
  may differ from the oracle's only if the oracle's own surface has the two cells within
  2 delta_c of each other (a near-tie: no FP32 evaluation can be expected to order them);
* refined surface: delta_r likewise over the Cf^2 refined placements, and the zoomed surface
  Zm = U G U^T (the intent of lib/libampcor_cuda/correlators/Sequential.icc:1101-1286) moves by
  at most delta_z = L^2 delta_r + 1e-6 |Zm|max, L the largest absolute row sum of U (a bound of
  the linear map) and 1e-6 the 3xTF32 / FP32 arithmetic of the zoom itself; the GPU's zoom cell
  may differ from the oracle's only if the oracle's zoomed surface has the two cells within
  2 delta_z;
* where the cells agree, the offsets must be equal to the oracle's float32 offsets bit for bit;
* peak correlation (the refined maximum) within 1e-5 relative of the oracle;
* every surface within ``surf_atol`` of the oracle (so every delta is small by itself).

A pair whose cells differ but whose bound does not explain it is a failure.  Near-ties (pairs
whose oracle top-two gap lies within twice their bound) are flagged and counted whether or not
the GPU's cell differs.
"""
from __future__ import annotations

import time

import numpy as np

import oracle

PEAK_RTOL = 1e-5
SURF_ATOL = 2e-5
ZOOM_ARITH = 1e-6


def oracle_run(ref, tgt, ulhc, R, W, f, m, z, deramp=False, threads=None):
    """The oracle's full pipeline with surfaces, and the restated reference CPU correlator's
    integer argmax; a dict reusable across forms."""
    t0 = time.perf_counter()
    off, od, cs, rs = oracle.adjust(ref, tgt, ulhc, R, W, f, m, z, surfaces=True,
                                    threads=threads, deramp=deramp)
    adjust_s = time.perf_counter() - t0
    arg, gap = oracle.coarse_cpu(ref, tgt, ulhc, R, W, threads=threads)
    return dict(offsets=off, diag=od, coarse=cs, refined=rs, cpu_arg=arg, cpu_gap=gap,
                geometry=(R, W, f, m, z), adjust_seconds=adjust_s)


def _zoom_at(U, G, p, q):
    """Zm[p, q] = U[p] G U[q]^T per pair (vectors of cells)."""
    return np.einsum("pa,pab,pb->p", U[p], G, U[q])


def compare(orc, gpu_offsets, gpu_diag, gpu_coarse, gpu_refined, surf_atol=SURF_ATOL):
    """Check a GPU run against ``oracle_run``'s output pair by pair.  ``gpu_diag`` is the
    structured diagnostics array (coarse_u/v, top/left, fine_p/q, refined_peak, coarse_peak),
    the surfaces are (P, C, C) and (P, Cf, Cf) float arrays.  Returns a report dict whose
    ``failures`` lists every pair the rules above do not excuse."""
    R, W, f, m, z = orc["geometry"]
    od = orc["diag"]
    P = len(od)
    C, Cf = W - R + 1, 2 * f * m + 1
    cs_o = orc["coarse"].reshape(P, C * C)
    rs_o = orc["refined"].reshape(P, Cf * Cf)
    cs_g = np.asarray(gpu_coarse, np.float64).reshape(P, C * C)
    rs_g = np.asarray(gpu_refined, np.float64).reshape(P, Cf * Cf)
    d = gpu_diag
    rows = np.arange(P)
    failures = []

    # the restated reference CPU correlator (uncentred chip, A.11) and the intended NCC share
    # their argmax; both FP64, so only an FP64 near-tie could split them
    cpu_same = (orc["cpu_arg"][:, 0] == od["coarse_u"]) & (orc["cpu_arg"][:, 1] == od["coarse_v"])
    cpu_split = np.flatnonzero(~cpu_same & (orc["cpu_gap"] > 1e-9))
    for p in cpu_split:
        failures.append((int(p), "oracle: reference CPU argmax differs from the intended NCC"))

    # coarse cell
    dc = np.abs(cs_g - cs_o).max(axis=1)
    ko = od["coarse_u"].astype(np.int64) * C + od["coarse_v"]
    kg = d["coarse_u"].astype(np.int64) * C + d["coarse_v"]
    coarse_flag = od["coarse_gap"] <= 2.0 * dc
    coarse_diff = kg != ko
    gap_at = cs_o[rows, ko] - cs_o[rows, np.clip(kg, 0, C * C - 1)]
    for p in np.flatnonzero(coarse_diff):
        if not (0 <= kg[p] < C * C) or gap_at[p] > 2.0 * dc[p]:
            failures.append((int(p), f"coarse cell {int(kg[p])} != {int(ko[p])}, gap "
                                     f"{gap_at[p]:.3g} > 2 x {dc[p]:.3g}"))
    same = ~coarse_diff
    for p in np.flatnonzero(same & ((d["top"] != od["top"]) | (d["left"] != od["left"]))):
        failures.append((int(p), "nudged corner differs"))

    # refined surface and zoom cell, on the pairs with the oracle's coarse cell
    dr = np.abs(rs_g - rs_o).max(axis=1)
    U = oracle.interp_matrix(Cf, z)
    L = np.abs(U).sum(axis=1).max()
    G = rs_o.reshape(P, Cf, Cf)
    zpeak = np.abs(od["zoom_peak"])
    dz = L * L * dr + ZOOM_ARITH * np.maximum(zpeak, 1.0)
    zoom_flag = same & (od["zoom_gap"] <= 2.0 * dz)
    fp, fq = d["fine_p"].astype(np.int64), d["fine_q"].astype(np.int64)
    op, oq = od["fine_p"].astype(np.int64), od["fine_q"].astype(np.int64)
    zoom_diff = same & ((fp != op) | (fq != oq))
    Z = z * Cf
    idx = np.flatnonzero(zoom_diff)
    if len(idx):
        inb = (fp[idx] >= 0) & (fp[idx] < Z) & (fq[idx] >= 0) & (fq[idx] < Z)
        zg = np.full(len(idx), -np.inf)
        ok = idx[inb]
        zg[inb] = _zoom_at(U, G[ok], fp[ok], fq[ok])
        zo = _zoom_at(U, G[idx], op[idx], oq[idx])
        for k, p in enumerate(idx):
            if zo[k] - zg[k] > 2.0 * dz[p]:
                failures.append((int(p), f"zoom cell ({fp[p]},{fq[p]}) != ({op[p]},{oq[p]}), gap "
                                         f"{zo[k] - zg[k]:.3g} > 2 x {dz[p]:.3g}"))
    exact = same & ~zoom_diff
    off_g = np.asarray(gpu_offsets, np.float32).reshape(P, 2)
    off_o = orc["offsets"]
    for p in np.flatnonzero(exact & ~(off_g == off_o).all(axis=1)):
        failures.append((int(p), f"offsets {off_g[p]} != oracle {off_o[p]} on the same cells"))

    # peak correlation and surfaces
    rel = np.abs(d["refined_peak"] - od["refined_peak"]) / np.maximum(np.abs(od["refined_peak"]), 1e-30)
    for p in np.flatnonzero(same & (rel > PEAK_RTOL)):
        failures.append((int(p), f"refined peak relative error {rel[p]:.3g}"))
    for p in np.flatnonzero(dc > surf_atol):
        failures.append((int(p), f"coarse surface error {dc[p]:.3g}"))
    for p in np.flatnonzero(same & (dr > surf_atol)):
        failures.append((int(p), f"refined surface error {dr[p]:.3g}"))

    err = np.abs(off_g.astype(np.float64) - off_o.astype(np.float64)).max(axis=1)
    failing = np.zeros(P, bool)
    failing[[fp_ for fp_, _ in failures]] = True
    excused = (coarse_diff | zoom_diff) & ~failing
    return {
        "pairs_checked": int(P),
        "failures": failures,
        "coarse_cells_differing": int(coarse_diff.sum()),
        "zoom_cells_differing": int(zoom_diff.sum()),
        "pairs_excused": int(excused.sum()),
        "near_ties_flagged": int((coarse_flag | zoom_flag).sum()),
        "max_abs_err_vs_oracle_px": float(np.nanmax(err)) if P else 0.0,
        "max_abs_err_non_excused_px": float(np.nanmax(err[~excused])) if (~excused).any() else 0.0,
        "failing_pairs": int(failing.sum()),
        "max_coarse_surface_err": float(dc.max()) if P else 0.0,
        "max_refined_surface_err": float(dr[same].max()) if same.any() else 0.0,
        "max_peak_rel_err": float(rel[same].max()) if same.any() else 0.0,
        "zoom_bound_lipschitz": float(L),
    }


def summary(rep):
    """The report without the failure list, plus its first few failures."""
    out = {k: v for k, v in rep.items() if k != "failures"}
    out["failures"] = len(rep["failures"])
    out["first_failures"] = rep["failures"][:5]
    return out
