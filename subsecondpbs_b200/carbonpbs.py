"""CarbonPBS-contract entry points of the reference's pybind module: cuFinalDose,
calcDose and cuCalDose (one function under three names), cuCalDose3 and
debug_build_carbonpbs_context (src/bindings/raytracedicom_pybind.cpp:1121-1636,
1873-2053, 2088-2313).

A CarbonPBS export (the rayweq volume with its 9-value header, spot coordinates
on the rayweq texel grid, an IDD table, the subspot table, per-spot directions
and cut-offs) is turned into one beam and one set of lookup tables, and the dose
runs through the library's wrapper (pbs_subsecond_wrapper) with the rayweq
volume as the transport. The CT handed to the wrapper only fixes the dose grid
geometry: 1000 (HU+1000 water) everywhere, or 1000 on the ROI voxels and 0
elsewhere when an ROI is given, as the reference builds it.

Argument names, their meaning, the accepted shapes and the error messages follow
the reference. Deviations: a (Nx, Ny, Nz) output array is accumulated onto its
own values like the other layouts (the reference accumulates it onto an
uninitialised buffer, raytracedicom_pybind.cpp:987-991); cuCalDose3's dose grid
starts at zero for the same reason; when `tables_dir` holds no reference tables
the density / stopping-power / radiation-length tables and the nuclear halo
tables come from the package's synthetic set (subsecondpbs_b200.tables).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import _lib

__all__ = ["cuFinalDose", "calcDose", "cuCalDose", "cuCalDose3", "debug_build_carbonpbs_context",
           "build_carbonpbs_context", "roi_linear_indices", "energy_from_carbonpbs"]


# ---- array conversions (raytracedicom_pybind.cpp:46-258) -----------------------

def _floats(obj) -> np.ndarray:
    a = np.asarray(obj, dtype=np.float32)
    if a.ndim == 0:
        return a.reshape(1)
    if a.ndim != 1 and not (a.ndim == 2 and (a.shape[0] == 1 or a.shape[1] == 1)):
        raise RuntimeError("Expected 1D float array or vector-like 2D float array")
    return np.ascontiguousarray(a.reshape(-1))


def _ints(obj) -> np.ndarray:
    a = np.asarray(obj)
    if a.ndim != 1 and not (a.ndim == 2 and (a.shape[0] == 1 or a.shape[1] == 1)):
        raise RuntimeError("Expected 1D int array")
    return np.ascontiguousarray(a.reshape(-1).astype(np.int32))


def _columns(obj, width: int, expected: int = 0) -> np.ndarray:
    """(N, width), (width, N) or flat arrays as a flat [N][width] float array."""
    a = np.asarray(obj, dtype=np.float32)
    if a.ndim == 1:
        if a.size % width:
            raise RuntimeError(f"Expected flattened {width}-vector array with length multiple of {width}")
        out = a
    elif a.ndim == 2:
        if a.shape[1] == width:
            out = a
        elif a.shape[0] == width:
            out = a.T
        else:
            raise RuntimeError(f"Expected shape (N,{width}) or ({width},N) for {width}-vector array")
    else:
        raise RuntimeError("Expected 1D or 2D float array")
    out = np.ascontiguousarray(out.reshape(-1))
    if expected > 0 and out.size != expected * width:
        raise RuntimeError(f"{width}-vector array length does not match expected count")
    return out


def _vec3(obj) -> tuple:
    a = np.asarray(obj, dtype=np.float32)
    if a.ndim == 1 and a.size >= 3:
        return tuple(float(v) for v in a[:3])
    if a.ndim == 2 and a.shape[0] == 3 and a.shape[1] >= 1:
        return tuple(float(v) for v in a[:, 0])
    if a.ndim == 2 and a.shape[1] == 3 and a.shape[0] >= 1:
        return tuple(float(v) for v in a[0, :3])
    raise RuntimeError("Expected 3-vector input")


def _mean_direction(dirs: np.ndarray) -> tuple:
    if dirs.size == 0 or dirs.size % 3:
        raise RuntimeError("Direction array must contain one or more 3-vectors")
    m = dirs.reshape(-1, 3).astype(np.float64).mean(axis=0).astype(np.float32)
    n = np.float32(np.sqrt(np.float32(m[0] * m[0] + m[1] * m[1] + m[2] * m[2])))
    if n > 0:
        m = m / n
    return tuple(float(v) for v in m)


def roi_linear_indices(roi, dims) -> np.ndarray:
    """ROI voxels as linear indices x*ny*nz + y*nz + z (raytracedicom_pybind.cpp:
    856-933): flat linear indices, flat xyz triplets (when every triplet is inside
    the grid), or (N,3) / (3,N) arrays."""
    nx, ny, nz = (int(v) for v in dims)
    a = np.asarray(roi)
    if a.ndim == 1:
        v = a.astype(np.int32)
        if v.size and v.size % 3 == 0:
            t = v.reshape(-1, 3)
            if ((t[:, 0] >= 0) & (t[:, 0] < nx) & (t[:, 1] >= 0) & (t[:, 1] < ny) & (t[:, 2] >= 0) &
                    (t[:, 2] < nz)).all():
                return (t[:, 0] * ny * nz + t[:, 1] * nz + t[:, 2]).astype(np.int32)
        return v
    if a.ndim != 2:
        raise RuntimeError("roi_index must be 1D xyz triplets or 2D (N,3)/(3,N)")
    a = a.astype(np.int32)
    if a.shape[1] == 3:
        return (a[:, 0] * ny * nz + a[:, 1] * nz + a[:, 2]).astype(np.int32)
    if a.shape[0] == 3:
        return (a[0] * ny * nz + a[1] * nz + a[2]).astype(np.int32)
    raise RuntimeError("roi_index must have shape (N,3) or (3,N)")


def _slice_mode(env: str) -> str:
    v = os.environ.get(env, "").strip().lower()
    if v in ("head", "prefix"):
        return "head"
    return "tail"


def _slice(energies: np.ndarray, rows: int, mode: str) -> np.ndarray:
    if rows <= 0 or energies.size == 0:
        return energies[:0]
    keep = min(energies.size, rows)
    return energies[:keep] if mode == "head" else energies[energies.size - keep:]


# ---- lookup tables (raytracedicom_pybind.cpp:459-638, nuclear_table_utils.h) ---

def _reference_tables(tables_dir) -> dict:
    from .tables import energy_reader, synthetic_nuclear_tables, synthetic_proton_tables

    d = Path(tables_dir) if tables_dir is not None else None
    if d is not None and (d / "density_Schneider2000_adj.txt").exists():
        try:
            return energy_reader(d, nuclear=True)
        except (OSError, ValueError):
            return energy_reader(d)
    return synthetic_nuclear_tables(synthetic_proton_tables())


def _frac_index(xs: np.ndarray, x: float) -> float:
    """findFractionalIndexMonotonic (nuclear_table_utils.h:24-60)."""
    n = xs.size
    if n <= 1:
        return 0.0
    if xs[-1] >= xs[0]:
        if x <= xs[0]:
            return 0.0
        if x >= xs[-1]:
            return float(n - 1)
        for i in range(1, n):
            if x <= xs[i]:
                den = np.float32(xs[i] - xs[i - 1])
                t = np.float32(x - xs[i - 1]) / den if abs(den) > 1e-12 else np.float32(0)
                return float(np.float32(i - 1) + min(np.float32(1), max(np.float32(0), t)))
    else:
        if x >= xs[0]:
            return 0.0
        if x <= xs[-1]:
            return float(n - 1)
        for i in range(1, n):
            if x >= xs[i]:
                den = np.float32(xs[i] - xs[i - 1])
                t = np.float32(x - xs[i - 1]) / den if abs(den) > 1e-12 else np.float32(0)
                return float(np.float32(i - 1) + min(np.float32(1), max(np.float32(0), t)))
    return float(n - 1)


def _row_linear(m: np.ndarray, row: int, idx: np.ndarray) -> np.ndarray:
    cols = m.shape[1]
    c = np.clip(idx, 0.0, cols - 1).astype(np.float32)
    i0 = np.floor(c).astype(np.int64)
    fr = (c - i0).astype(np.float32)
    i1 = np.minimum(cols - 1, i0 + (fr > 0))
    v0, v1 = m[row, i0], m[row, i1]
    return (v0 + (v1 - v0) * fr).astype(np.float32)


def _align_nuclear(ref: dict, out: dict) -> None:
    """The reference tables' nuclear weight / sigma^2 resampled onto `out`'s energy
    and depth axes (alignNuclearTablesToPrimaryAxis, nuclear_table_utils.h:125-189)."""
    if "nuc_weight_matrix" not in ref or "nuc_sq_sigma_matrix" not in ref:
        return
    rw = np.asarray(ref["nuc_weight_matrix"], np.float32).reshape(ref["n_energies"], ref["n_energy_samples"])
    rs = np.asarray(ref["nuc_sq_sigma_matrix"], np.float32).reshape(ref["n_energies"], ref["n_energy_samples"])
    ne, ns = out["n_energies"], out["n_energy_samples"]
    re_, rsf = np.asarray(ref["energies_per_u"], np.float32), np.asarray(ref["scale_facts"], np.float32)
    same = (ref["n_energies"] == ne and ref["n_energy_samples"] == ns and
            np.allclose(re_, out["energies_per_u"], atol=1e-4) and
            np.allclose(ref["peak_depths"], out["peak_depths"], atol=1e-4) and
            np.allclose(rsf, out["scale_facts"], atol=1e-4))
    if same:
        w, s = rw.copy(), rs.copy()
    else:
        w = np.zeros((ne, ns), np.float32)
        s = np.zeros((ne, ns), np.float32)
        j = np.arange(ns, dtype=np.float32)
        for e in range(ne):
            ei = _frac_index(re_, float(out["energies_per_u"][e]))
            e_int = int(np.floor(ei))
            fr = np.float32(ei - e_int)
            e0 = max(0, min(ref["n_energies"] - 1, e_int))
            e1 = max(0, min(ref["n_energies"] - 1, e0 + (1 if fr > 0 else 0)))
            ts = np.float32(out["scale_facts"][e])
            depth = j / ts if ts > 0 else np.zeros_like(j)
            w0, w1 = _row_linear(rw, e0, depth * rsf[e0]), _row_linear(rw, e1, depth * rsf[e1])
            s0, s1 = _row_linear(rs, e0, depth * rsf[e0]), _row_linear(rs, e1, depth * rsf[e1])
            w[e] = w0 + (w1 - w0) * fr
            s[e] = s0 + (s1 - s0) * fr
    out["nuc_weight_matrix"] = w
    out["nuc_sq_sigma_matrix"] = s
    out["nuclear_tables_aligned_to_primary_axis"] = True


def energy_from_carbonpbs(enelist, idddata, iddsetting, tables_dir="tables/") -> dict:
    """Lookup tables from a CarbonPBS IDD table (build_energy_from_carbonpbs,
    raytracedicom_pybind.cpp:521-638): CIDD = running sum of IDD * step, one depth
    scale per energy (1 / step), peak depth at each row's maximum; the depth unit
    is taken as cm (x10) for short steps and short spans; density, stopping-power
    and radiation-length tables come from `tables_dir`."""
    energies = _floats(enelist)
    if energies.size == 0:
        raise RuntimeError("enelist must not be empty")
    setting = _floats(iddsetting)
    if setting.size < 3:
        raise RuntimeError("iddsetting must provide [start, step, nSamples]")
    idd = np.asarray(idddata, dtype=np.float32)
    if idd.ndim != 2:
        raise RuntimeError("idddata must be a 2D array with shape (n_energies, n_samples)")
    rows, cols = idd.shape
    if rows <= 0 or rows > energies.size:
        raise RuntimeError("idddata rows must be in the range [1, enelist length]")
    if rows != energies.size:
        energies = _slice(energies, rows, _slice_mode("RTD_IDD_SLICE_MODE"))
    start_raw, step_raw = np.float32(setting[0]), np.float32(setting[1])
    logical = int(np.rint(setting[2]))
    compacted = cols > 0 and logical > cols
    depth_scale = np.float32(logical) / np.float32(cols) if compacted else np.float32(1)
    unit = np.float32(1)
    span = np.float32((cols - 1) * step_raw * depth_scale) if cols > 1 else np.float32(step_raw * depth_scale)
    max_e = float(energies.max())
    if not compacted and 0 < step_raw < 1 and span < 20:
        unit = np.float32(10)
    elif not compacted and max_e >= 250 and 20 < span <= 100:
        unit = np.float32(10)
    start = np.float32(start_raw * unit)
    step = np.float32(step_raw * depth_scale * unit)
    scale = np.float32(1) / step if step > 0 else np.float32(1)
    cidd = np.cumsum(idd * step, axis=1, dtype=np.float32)
    ref = _reference_tables(tables_dir)
    finite = np.where(np.isfinite(idd), idd, -np.inf)
    peaks = (start + step * np.argmax(finite, axis=1).astype(np.float32)).astype(np.float32)
    if not (peaks > 0).any():
        re_, rp = np.asarray(ref["energies_per_u"], np.float32), np.asarray(ref["peak_depths"], np.float32)
        order = np.argsort(re_)
        peaks = np.interp(energies, re_[order], rp[order]).astype(np.float32)
    out = {"n_energies": int(rows), "n_energy_samples": int(cols), "energies_per_u": energies.astype(np.float32),
           "peak_depths": peaks, "scale_facts": np.full(rows, scale, np.float32), "cidd_matrix": cidd}
    for key in ("density", "sp", "rrl"):
        out[f"{key}_vector"] = ref[f"{key}_vector"]
        out[f"n_{key}_samples"] = ref[f"n_{key}_samples"]
        out[f"{key}_scale_fact"] = ref[f"{key}_scale_fact"]
    _align_nuclear(ref, out)
    return out


# ---- beam (raytracedicom_pybind.cpp:640-757, 1121-1373) -------------------------

def _layer_cutoffs(per_spot: np.ndarray, counts: np.ndarray) -> np.ndarray:
    out, off = [], 0
    for layer, c in enumerate(counts):
        c = max(0, int(c))
        cut = 0.0
        if c > 0 and off < per_spot.size:
            cut = float(per_spot[off])
        for i in range(c):
            idx = off + i
            if idx >= per_spot.size:
                break
            if abs(float(per_spot[idx]) - cut) > 1e-3:
                raise RuntimeError(
                    f"longitudal_cutoff varies within layer {layer}: first={cut:f}, current={float(per_spot[idx]):f}, "
                    f"spot_offset={i}. Current RTD compatibility path only supports one longitudinal cutoff per layer.")
        out.append(cut)
        off += c
    return np.asarray(out, np.float32)


def _remap_subspots(lut_energies, lut_sub, lut_sig, energies):
    """Subspot table rows and sigmas interpolated from the LUT energies to the
    layer energies (remap_subspot_lut_to_actual_layers)."""
    n_lut, m = lut_sub.shape[0], lut_sub.shape[1]
    sub = np.zeros((energies.size, m, 5), np.float32)
    sig = np.zeros((energies.size, 2), np.float32)
    if n_lut <= 0 or m <= 0 or lut_energies.size == 0:
        return sub, sig
    asc = lut_energies[0] <= lut_energies[-1]
    lo, hi = (lut_energies[0], lut_energies[-1]) if asc else (lut_energies[-1], lut_energies[0])
    for layer, e in enumerate(energies):
        if e <= lo:
            idx = 0.0 if asc else float(lut_energies.size - 1)
        elif e >= hi:
            idx = float(lut_energies.size - 1) if asc else 0.0
        else:
            idx = float(lut_energies.size - 1) if asc else 0.0
            for i in range(lut_energies.size - 1):
                a, b = lut_energies[i], lut_energies[i + 1]
                if e < min(a, b) or e > max(a, b):
                    continue
                den = np.float32(b - a)
                t = np.float32(e - a) / den if abs(den) > 1e-6 else np.float32(0)
                idx = float(np.float32(i) + min(np.float32(1), max(np.float32(0), t)))
                break
        i_int = int(np.floor(idx))
        fr = np.float32(idx - i_int)
        i0 = max(0, min(n_lut - 1, i_int))
        i1 = max(0, min(n_lut - 1, i0 + (1 if fr > 0 else 0)))
        sub[layer] = lut_sub[i0] + (lut_sub[i1] - lut_sub[i0]) * fr
        s0, s1 = lut_sig[min(i0, lut_sig.shape[0] - 1)], lut_sig[min(i1, lut_sig.shape[0] - 1)]
        sig[layer] = s0 + (s1 - s0) * fr
    return sub, sig


def build_carbonpbs_context(rayweq, roiIdx, all_energies, sourcePos, tmpBeamDir, bmxdir, bmydir, corner, resolution,
                            dims, longitudalCutoff, enelist, idddata, iddsetting, profiledata, profilesetting,
                            beamparadata, subspotdata, layerInfo, layerEnergy, idbeamxy, nPar, sad,
                            beamParaPos=None, tables_dir="tables/") -> dict:
    """{'dims', 'corner', 'resolution', 'beam', 'energy'} of a CarbonPBS export
    (build_carbonpbs_context, raytracedicom_pybind.cpp:1121-1373)."""
    d = [int(v) for v in np.asarray(dims).reshape(-1)]
    if len(d) != 3:
        raise RuntimeError("dims must contain exactly 3 integers")
    corner_v, res_v = _floats(corner), _floats(resolution)
    if corner_v.size != 3 or res_v.size != 3:
        raise RuntimeError("corner and resolution must contain exactly 3 floats")
    spot_energies = _floats(all_energies) if np.asarray(all_energies).size else np.zeros(0, np.float32)
    lut_energies = _floats(enelist)
    weq = np.ascontiguousarray(np.asarray(rayweq, dtype=np.float32).reshape(-1))
    if weq.size < 9:
        raise RuntimeError("rayweq must include the 9-value CarbonPBS header")
    header = weq[:9].copy()
    weights = _floats(nPar)
    counts = _ints(layerInfo)
    energies = _floats(layerEnergy)
    if spot_energies.size and spot_energies.size != weights.size:
        raise RuntimeError("all_energies length must match nPar length")
    dirs = _columns(tmpBeamDir, 3, weights.size)
    sad_a = np.asarray(sad, dtype=np.float32).reshape(-1)
    if sad_a.size == 0:
        raise RuntimeError("sad array must not be empty")
    sad_v = float(sad_a[0])
    beam = {
        "water_equivalence": weq,
        "ray_weq_header": header,
        "ray_spacing": (float(header[7]), float(header[4])),
        # The physical spot spacing is not part of the export: the planner infers it.
        "spot_delta": (0.0, 0.0, 0.0),
        "steps": max(1, int(np.rint(header[2]))),
        "roi_linear_indices": roi_linear_indices(roiIdx, d),
        "energies": energies,
        "layer_spot_counts": counts,
        "spot_weights": weights,
        "spot_positions": _columns(idbeamxy, 2, weights.size),
        "spot_positions_are_indices": True,
        "spot_beam_directions": dirs,
        "beam_direction": _mean_direction(dirs),
        "beam_xdir": _vec3(bmxdir),
        "beam_ydir": _vec3(bmydir),
        "source_position": tuple(float(v) for v in _columns(sourcePos, 3)[:3]),
        "ref_plane_z": 0.0,
        "sad": sad_v,
        "source_dist": (0.0, 0.0),
        "spot_offset": (0.0, 0.0, 0.0),
    }
    if longitudalCutoff is not None:
        per_spot = _floats(longitudalCutoff) if np.asarray(longitudalCutoff).size else np.zeros(0, np.float32)
        if per_spot.size:
            if per_spot.size != int(counts.sum()):
                raise RuntimeError("longitudal_cutoff length must match total spot count")
            beam["layer_longitudinal_cutoffs"] = _layer_cutoffs(per_spot, counts)
    prof_rows = 0
    if profiledata is not None:
        prof = np.asarray(profiledata, dtype=np.float32)
        beam["profile_data"] = prof.reshape(-1)
        prof_rows = int(prof.shape[0]) if prof.ndim >= 1 else 0
        depth_n = prof.shape[1] if prof.ndim >= 2 else 0
        if profilesetting is not None:
            ps = _floats(profilesetting).copy()
            if ps.size >= 3 and depth_n > 0:
                logical = max(0, int(np.rint(ps[2])))
                if logical > depth_n:
                    ps[1] *= np.float32(logical) / np.float32(depth_n)
                ps[2] = np.float32(depth_n)
            beam["profile_setting"] = ps
    elif profilesetting is not None:
        beam["profile_setting"] = _floats(profilesetting)
    # The profile rows' energy axis: the machine energy list, sliced to the row count
    # when they differ (raytracedicom_pybind.cpp:1291-1294, RTD_PROFILE_SLICE_MODE).
    beam["profile_energies"] = lut_energies
    if prof_rows > 0 and lut_energies.size and prof_rows != lut_energies.size:
        beam["profile_energies"] = _slice(lut_energies, prof_rows, _slice_mode("RTD_PROFILE_SLICE_MODE"))
    if beamparadata is not None:
        beam["beam_para_data"] = np.asarray(beamparadata, dtype=np.float32).reshape(-1)
    if beamParaPos is not None:
        beam["beam_para_pos"] = float(np.asarray(beamParaPos, dtype=np.float32).reshape(-1)[0])
    sub = np.asarray(subspotdata, dtype=np.float32)
    if sub.ndim != 3 or sub.shape[2] != 5:
        raise RuntimeError("subspotdata must have shape (num_layers, max_subspots_per_layer, 5)")
    if counts.size != energies.size:
        raise RuntimeError("layerEnergy/layerInfo size mismatch")
    energy = energy_from_carbonpbs(enelist, idddata, iddsetting, tables_dir)
    lut_sig = sub[:, 0, 3:5].copy()
    if sub.shape[0] == energies.size:
        beam["subspot_data"], beam["spot_sigmas"] = sub, lut_sig
    else:
        beam["subspot_data"], beam["spot_sigmas"] = _remap_subspots(lut_energies, sub, lut_sig, energies)
    return {"dims": d, "corner": tuple(float(v) for v in corner_v), "resolution": tuple(float(v) for v in res_v),
            "beam": beam, "energy": energy, "beam_para_pos": beamParaPos}


def debug_build_carbonpbs_context(rayweq, roiIdx, all_energies, sourcePos, tmpBeamDir, bmxdir, bmydir, corner,
                                  resolution, dims, longitudalCutoff, enelist, idddata, iddsetting, profiledata,
                                  profilesetting, beamparadata, subspotdata, layerInfo, layerEnergy, idbeamxy, nPar,
                                  sad, beamParaPos=None, tables_dir="tables/") -> dict:
    """The converted context's bookkeeping without running the dose
    (raytracedicom_pybind.cpp:1375-1467)."""
    ctx = build_carbonpbs_context(rayweq, roiIdx, all_energies, sourcePos, tmpBeamDir, bmxdir, bmydir, corner,
                                  resolution, dims, longitudalCutoff, enelist, idddata, iddsetting, profiledata,
                                  profilesetting, beamparadata, subspotdata, layerInfo, layerEnergy, idbeamxy, nPar,
                                  sad, beamParaPos, tables_dir)
    b, e = ctx["beam"], ctx["energy"]
    roi = b["roi_linear_indices"]
    out = {
        "dims": list(ctx["dims"]), "rayWeqHeader": [float(v) for v in b["ray_weq_header"]],
        "weq_len": int(b["water_equivalence"].size), "layer_energies": [float(v) for v in b["energies"]],
        "layerSpotCounts": [int(v) for v in b["layer_spot_counts"]], "totalSpots": int(b["layer_spot_counts"].sum()),
        "spotPositions": int(b["spot_positions"].size // 2), "spotWeights": int(b["spot_weights"].size),
        "spotDirections": int(b["spot_beam_directions"].size // 3), "spotPositionsAreIndices": True,
        "subspotDataSize": int(np.asarray(b["subspot_data"]).size),
        "maxSubspotsPerLayer": int(np.asarray(b["subspot_data"]).shape[1]), "roiLinearIndices": int(roi.size),
        "sourcePosition": list(b["source_position"]), "sad": b["sad"],
        "profileSettingSize": int(np.asarray(b.get("profile_setting", [])).size),
        "beamParaDataSize": int(np.asarray(b.get("beam_para_data", [])).size),
        "energyData_nEnergies": e["n_energies"], "energyData_nEnergySamples": e["n_energy_samples"],
        "energyData_ciddMatrixSize": int(np.asarray(e["cidd_matrix"]).size),
    }
    if roi.size:
        out["roiLinearMin"], out["roiLinearMax"] = int(roi.min()), int(roi.max())
    return out


# ---- running the dose (raytracedicom_pybind.cpp:935-1081, 1469-1676) -------------

def _ct_for(dims, roi) -> np.ndarray:
    n = int(np.prod(dims))
    if roi.size == 0:
        return np.full(n, 1000.0, np.float32)
    ct = np.zeros(n, np.float32)
    ok = roi[(roi >= 0) & (roi < n)]
    ct[ok] = 1000.0
    return ct


def _run(final_dose, ct, ctx, gpu_id, nuclear, verbose):
    dims = ctx["dims"]
    out = final_dose
    if not isinstance(out, np.ndarray) or out.dtype != np.float32:
        raise RuntimeError("out_final_dose must be a float32 numpy array")
    n = int(np.prod(dims))
    if out.size != n:
        raise RuntimeError("out_final_dose size does not match dims")
    if ct.size != n:
        raise RuntimeError("ct_data size does not match dims")
    if out.ndim == 1:
        work, commit = out, None
    elif out.ndim == 3 and out.flags.c_contiguous and tuple(out.shape) == (dims[0], dims[1], dims[2]):
        work = np.ascontiguousarray(out.transpose(2, 1, 0))
        commit = "xyz"
    elif out.ndim == 3 and out.flags.c_contiguous and tuple(out.shape) == (dims[2], dims[1], dims[0]):
        work, commit = out, None
    else:
        raise RuntimeError(
            "out_final_dose must be either 1D flat, C-contiguous (Nz,Ny,Nx), or C-contiguous (Nx,Ny,Nz)")
    if not work.flags.c_contiguous:
        raise RuntimeError("out_final_dose must be C-contiguous")
    from .cudaCalDoseRTD import _with_luts

    lib = _lib.load()
    bd, kb = _lib.beam_desc(ctx["beam"])
    ed, ke = _lib.energy_desc(_with_luts(ctx["energy"], None))
    fp = C.POINTER(C.c_float)
    ctc = np.ascontiguousarray(ct, dtype=np.float32)
    rc = lib.pbs_subsecond_wrapper(ctc.ctypes.data_as(fp), _lib.int3(dims), _lib.float3(ctx["resolution"]),
                                   _lib.float3(ctx["corner"]), work.ctypes.data_as(fp), _lib.int3(dims),
                                   _lib.float3(ctx["resolution"]), _lib.float3(ctx["corner"]), C.byref(bd), 1,
                                   C.byref(ed), int(gpu_id), int(bool(nuclear)), int(verbose))
    _lib.check(rc)
    del kb, ke
    if commit == "xyz":
        out[...] = work.transpose(2, 1, 0)
    vals = out.reshape(-1)
    if not np.isfinite(vals).all():
        raise RuntimeError("cuFinalDose/calcDose/cuCalDose produced NaN/Inf dose output")
    if (np.asarray(ctx["beam"]["spot_weights"]) > 0).any() and not (np.abs(vals) > 1e-20).any():
        raise RuntimeError("cuFinalDose/calcDose/cuCalDose produced an empty dose grid under positive spot weights; "
                           "wrapper execution likely failed or returned placeholder zeros")
    return final_dose


def cuFinalDose(finalDose, rayweq, roiIdx, all_energies, sourcePos, tmpBeamDir, bmxdir, bmydir, corner, resolution,
                dims, longitudalCutoff, enelist, idddata, iddsetting, profiledata, profilesetting, beamparadata,
                subspotdata, layerInfo, layerEnergy, idbeamxy, nPar, sad, cutoff=None, beamParaPos=None, gpuId=0,
                nuclear_correction=False, verbose=0, debug=False, tables_dir="tables/"):
    """Dose of one CarbonPBS-exported beam added into `finalDose` (float32, flat,
    (Nz,Ny,Nx) or (Nx,Ny,Nz)); returns `finalDose`. `cutoff` is accepted for the
    contract and not used, as in the reference (raytracedicom_pybind.cpp:1906)."""
    del cutoff, debug
    ctx = build_carbonpbs_context(rayweq, roiIdx, all_energies, sourcePos, tmpBeamDir, bmxdir, bmydir, corner,
                                  resolution, dims, longitudalCutoff, enelist, idddata, iddsetting, profiledata,
                                  profilesetting, beamparadata, subspotdata, layerInfo, layerEnergy, idbeamxy, nPar,
                                  sad, beamParaPos, tables_dir)
    ct = _ct_for(ctx["dims"], ctx["beam"]["roi_linear_indices"])
    return _run(finalDose, ct, ctx, gpuId, nuclear_correction, verbose)


calcDose = cuFinalDose
cuCalDose = cuFinalDose


def _influence(ctx, gpu_id, nuclear):
    """Dose-influence matrix of the export's spots on its (Nx, Ny, Nz) grid: scipy
    CSC of shape (voxels, spots) with rows as x-major linear indices
    (ix*Ny + iy)*Nz + iz, the CarbonPBS voxel order (deviceCalDose.cu:167-168)."""
    import scipy.sparse as sp

    from .cudaCalDoseRTD import DoseEngine

    dims = ctx["dims"]
    ct = _ct_for(dims, ctx["beam"]["roi_linear_indices"])
    eng = DoseEngine(gpu_id)
    try:
        eng.set_energy(ctx["energy"])
        eng.set_ct(ct.reshape(dims[2], dims[1], dims[0]), dims, ctx["resolution"], ctx["corner"])
        eng.set_dose_grid(dims, ctx["resolution"], ctx["corner"])
        a = eng.influence_csc(ctx["beam"], nuclear_correction=nuclear).tocoo()
    finally:
        eng.close()
    nx, ny, nz = dims
    v = a.row.astype(np.int64)
    x, y, z = v % nx, (v // nx) % ny, v // (nx * ny)
    rows = (x * ny + y) * nz + z
    return sp.csc_matrix((a.data, (rows, a.col)), shape=a.shape)


def cuCalDose3(out_cscdata, out_cscptr, out_cscrowind, weq_data, roi_index, source_energies, source, beam_dir,
               beam_xdir, beam_ydir, corner, resolution, dims, longitudal_cutoff, enelist, idddata, iddsetting,
               profiledata, profilesetting, beamparadata, subspot_data, layer_info, layer_energy, outNNZ, idbeamxy,
               num_particles_per_beam, cutoff, sad, beam_para_pos, python_nnz_size, gpu_id=0,
               nuclear_correction=False, verbose=0, tables_dir="tables/"):
    """The reference's cuCalDose3 (raytracedicom_pybind.cpp:1955-2053) computes the
    beam's dose into a new (Nx,Ny,Nz) grid and zeroes its sparse outputs; here the
    sparse outputs carry the spot-preserving dose-influence matrix the operator mode
    plans for (include/core/rtd_operator_mode.h:1-8), in the layout its CarbonPBS
    caller reads (tps_py/dosecal.py:1520-1530): `out_cscdata` / `out_cscrowind` hold
    the values and x-major voxel rows (ascending within a column), `out_cscptr[0]` = 0
    and `out_cscptr[1 + j]` the entry count of spot j (the caller takes the cumulative
    sum), `outNNZ[0]` the total. Columns are per unit spot weight (the matrix times
    num_particles_per_beam is the dose). Entries that do not fit the arrays (their
    capacity is their size) are not written; outNNZ still reports the total, as the
    caller's retry loop expects. Returns {'dose_grid', 'out_cscdata', 'out_cscptr',
    'out_cscrowind', 'outNNZ'}."""
    del cutoff, python_nnz_size
    for a in (out_cscdata, out_cscptr, out_cscrowind, outNNZ):
        if isinstance(a, np.ndarray) and a.size:
            if a.dtype not in (np.float32, np.int32, np.int64, np.uint64):
                raise RuntimeError("Unsupported dtype for zero fill")
            a[...] = 0
    d = [int(v) for v in np.asarray(dims).reshape(-1)]
    if len(d) != 3:
        raise RuntimeError("dims must contain exactly 3 integers")
    dose = np.zeros((d[0], d[1], d[2]), np.float32)
    ctx = build_carbonpbs_context(weq_data, roi_index, source_energies, source, beam_dir, beam_xdir, beam_ydir, corner,
                                  resolution, dims, longitudal_cutoff, enelist, idddata, iddsetting, profiledata,
                                  profilesetting, beamparadata, subspot_data, layer_info, layer_energy, idbeamxy,
                                  num_particles_per_beam, sad, beam_para_pos, tables_dir)
    ct = _ct_for(ctx["dims"], ctx["beam"]["roi_linear_indices"])
    _run(dose, ct, ctx, gpu_id, nuclear_correction, verbose)
    a = _influence(ctx, gpu_id, nuclear_correction)
    a.sort_indices()
    nnz = int(a.nnz)
    if isinstance(outNNZ, np.ndarray) and outNNZ.size:
        outNNZ.reshape(-1)[0] = nnz
    data, rowind, ptr = (np.asarray(v).reshape(-1) if isinstance(v, np.ndarray) else None
                         for v in (out_cscdata, out_cscrowind, out_cscptr))
    if ptr is not None and ptr.size >= a.shape[1] + 1:
        ptr[0] = 0
        ptr[1:a.shape[1] + 1] = np.diff(a.indptr)
    if data is not None and rowind is not None and nnz <= min(data.size, rowind.size):
        data[:nnz] = a.data
        rowind[:nnz] = a.indices
    return {"dose_grid": dose, "out_cscdata": out_cscdata, "out_cscptr": out_cscptr, "out_cscrowind": out_cscrowind,
            "outNNZ": outNNZ}


def cuCalDoseNorm(doseNorm, weqData, roiIndex, sourceEne, source, bmdir, bmxdir, bmydir, corner, resolution, dims,
                  longitudalCutoff, enelist, idddata, iddsetting, profiledata, profilesetting, beamparadata,
                  subSpotData, layerInfo, layerEnergy, idbeamxy, sad, cutoff, beamParaPos, gpuId=0,
                  nuclear_correction=False, tables_dir="tables/"):
    """CarbonPBS's cuCalDoseNorm (carbonPBS/cudaCalDose.cpp:347-500, registered at
    :1975, called by tps_py/dosecal.py:1504): `doseNorm[i]` = sum over the spots of
    the squared dose per unit spot weight at ROI voxel i (calDoseSumSquareKernel,
    carbonPBS/deviceCalDose.cu:123-229), the row norms of the dose-influence matrix.
    The ROI is given as in the other faces ((N,3), (3,N) or flat triplets, x-major
    layout); computed on the device without forming the matrix
    (pbs_context_influence_row_norms). Returns 1, the reference's success flag."""
    del cutoff
    from .cudaCalDoseRTD import DoseEngine

    d = [int(v) for v in np.asarray(dims).reshape(-1)]
    if len(d) != 3:
        raise RuntimeError("dims must contain exactly 3 integers")
    n_spots = np.asarray(idbeamxy).size // 2
    ctx = build_carbonpbs_context(weqData, roiIndex, sourceEne, source, bmdir, bmxdir, bmydir, corner, resolution,
                                  dims, longitudalCutoff, enelist, idddata, iddsetting, profiledata, profilesetting,
                                  beamparadata, subSpotData, layerInfo, layerEnergy, idbeamxy,
                                  np.ones(n_spots, np.float32), sad, beamParaPos, tables_dir)
    roi = ctx["beam"]["roi_linear_indices"]
    out = np.asarray(doseNorm).reshape(-1) if isinstance(doseNorm, np.ndarray) else None
    if out is None or out.dtype != np.float32 or out.size != roi.size:
        raise RuntimeError("doseNorm must be a float32 array with one entry per ROI voxel")
    nx, ny, nz = d
    ix, rem = roi // (ny * nz), roi % (ny * nz)
    iy, iz = rem // nz, rem % nz
    voxels = (iz.astype(np.int64) * ny + iy) * nx + ix
    ct = _ct_for(d, roi)
    eng = DoseEngine(gpuId)
    try:
        eng.set_energy(ctx["energy"])
        eng.set_ct(ct.reshape(nz, ny, nx), d, ctx["resolution"], ctx["corner"])
        eng.set_dose_grid(d, ctx["resolution"], ctx["corner"])
        out[...] = eng.influence_row_norms(ctx["beam"], voxels=voxels, nuclear_correction=nuclear_correction)
    finally:
        eng.close()
    return 1
