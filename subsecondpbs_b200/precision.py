"""Dose agreement figures used to state the error of a result against a
double-precision reference of the same inputs: the largest difference in units
of the reference maximum over voxels above 10 % of it, and the 1 %/1 mm global
gamma pass rate."""
from __future__ import annotations

import numpy as np


def max_rel_err(dose, ref, thr: float = 0.1) -> float:
    """max |dose - ref| / max(ref) over voxels where ref > thr * max(ref)."""
    ref = np.asarray(ref, np.float64)
    dmax = float(ref.max())
    mask = ref > thr * dmax
    return float(np.abs(np.asarray(dose, np.float64) - ref)[mask].max() / dmax)


def gamma_pass_rate(dose, ref, spacing_mm, dd: float = 0.01, dta_mm: float = 1.0, thr: float = 0.1) -> float:
    """1 %/1 mm global gamma over voxels above `thr` of Dmax; the evaluated dose is
    sampled at the voxel and at +-dta along each axis (linear interpolation).
    `spacing_mm` is (x, y, z) for arrays indexed [z][y][x]."""
    ref = np.asarray(ref, np.float64)
    ev = np.asarray(dose, np.float64)
    dmax = ref.max()
    mask = ref > thr * dmax
    best = ((ev - ref) / (dd * dmax)) ** 2
    for axis, sp in zip((2, 1, 0), spacing_mm):
        f = min(dta_mm / sp, 1.0)
        for sgn in (-1, 1):
            nb = np.roll(ev, -sgn, axis=axis)
            shifted = ev + f * (nb - ev)
            g = ((shifted - ref) / (dd * dmax)) ** 2 + (f * sp / dta_mm) ** 2
            best = np.minimum(best, g)
    return float((best[mask] <= 1.0).mean())


def report(dose, ref, spacing_mm) -> dict:
    """Both figures as a dict (the form bench.py and the serving reports use)."""
    return {"max_abs_err_frac_dmax": max_rel_err(dose, ref), "gamma_1pct_1mm": gamma_pass_rate(dose, ref, spacing_mm)}
