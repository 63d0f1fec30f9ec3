"""Lookup tables in the reference's text formats.

`energy_reader` parses the four whitespace-separated tables the reference loads
(src/utils/energy_reader.cpp:21-185):

  proton_cumul_ddd_data.txt    nSamples nEnergies, energies[nE], peakDepths[nE],
                               scaleFacts[nE], cidd[nE][nS]
  density_Schneider2000_adj.txt  n scale, density[n]   (index = (HU+1000)*scale)
  HU_to_SP_H&N_adj.txt           n scale, sp[n]        (index = (HU+1000)*scale)
  radiation_length.txt           n scale, rRl[n]       (index = density*scale)
  nuclear_weights_and_sigmas_fit.txt (optional) nS nE, energies, peaks, scales,
                               weight[nE][nS], sqSigma[nE][nS]

On the reference's own tables/ files the result is bit-identical to what the
reference's energyReader stores (decimal text to float32).

`save_table_npz` / `load_table_npz` keep a parsed energy dict as one compressed
numpy archive, so the tables can travel where the text files are not present.

`synthetic_proton_tables` / `synthetic_carbon_tables` generate tables of the same
layout from analytic models (Bragg-Kleeman range-energy relation with Gaussian
range straggling and a linear primary-fluence loss), so the pipeline can run
without the reference's data files. The dicts use the keys of the reference's
pybind energy dict (src/bindings/raytracedicom_pybind.cpp:1824-1847).
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

PROTON_FILE = "proton_cumul_ddd_data.txt"
DENSITY_FILE = "density_Schneider2000_adj.txt"
SP_FILE = "HU_to_SP_H&N_adj.txt"
RRL_FILE = "radiation_length.txt"
NUCLEAR_FILE = "nuclear_weights_and_sigmas_fit.txt"


def _read_numbers(path: Path) -> np.ndarray:
    return np.array(path.read_text().split(), dtype=np.float64)


def _read_lut(path: Path):
    v = _read_numbers(path)
    n = int(v[0])
    scale = float(v[1])
    if v.size < 2 + n:
        raise ValueError(f"{path}: expected {n} samples, found {v.size - 2}")
    return n, scale, v[2:2 + n].astype(np.float32)


NUCLEAR_FILES = {"GAUSS_FIT": NUCLEAR_FILE, "FLUKA": "nuclear_weights_and_sigmas_Fluka.txt",
                 "SOUKUP": "nuclear_weights_and_sigmas_Soukup.txt"}


def energy_reader(tables_dir: str | Path, nuclear: bool = False, nuclear_file: str = NUCLEAR_FILE) -> dict:
    """Parse the reference's LUT text files into the pybind energy dict.

    With `nuclear`, the halo weight and squared-sigma tables come from
    `nuclear_file` (the reference reads nuclear_weights_and_sigmas_fit.txt,
    energy_reader.cpp:136; the Fluka and Soukup files share its layout). Their
    energy, peak-depth and scale rows must agree with the proton file's within
    0.01, the reference's own check (energy_reader.cpp:148-167)."""
    d = Path(tables_dir)
    v = _read_numbers(d / PROTON_FILE)
    ns, ne = int(v[0]), int(v[1])
    o = 2
    energies = v[o:o + ne]; o += ne
    peaks = v[o:o + ne]; o += ne
    scales = v[o:o + ne]; o += ne
    if v.size < o + ns * ne:
        raise ValueError(f"{PROTON_FILE}: truncated CIDD matrix")
    cidd = v[o:o + ns * ne].reshape(ne, ns)
    out = {
        "n_energies": ne,
        "n_energy_samples": ns,
        "energies_per_u": energies.astype(np.float32),
        "peak_depths": peaks.astype(np.float32),
        "scale_facts": scales.astype(np.float32),
        "cidd_matrix": cidd.astype(np.float32),
    }
    for key, fname in (("density", DENSITY_FILE), ("sp", SP_FILE), ("rrl", RRL_FILE)):
        n, scale, vec = _read_lut(d / fname)
        out[f"n_{key}_samples"] = n
        out[f"{key}_scale_fact"] = scale
        out[f"{key}_vector"] = vec
    if nuclear:
        w = _read_numbers(d / nuclear_file)
        nns, nne = int(w[0]), int(w[1])
        if nns != ns or nne != ne:
            raise ValueError(f"{nuclear_file}: sample/energy counts differ from {PROTON_FILE}")
        for k, (name, ref) in enumerate((("energies", energies), ("peak depths", peaks), ("scale facts", scales))):
            row = w[2 + k * ne:2 + (k + 1) * ne].astype(np.float32)
            if np.any(np.abs(row - ref.astype(np.float32)) > 0.01):
                raise ValueError(f"{nuclear_file}: {name} differ from {PROTON_FILE}")
        o = 2 + 3 * ne
        if w.size < o + 2 * ns * ne:
            raise ValueError(f"{nuclear_file}: truncated weight/sigma matrices")
        out["nuc_weight_matrix"] = w[o:o + ns * ne].reshape(ne, ns).astype(np.float32)
        out["nuc_sq_sigma_matrix"] = w[o + ns * ne:o + 2 * ns * ne].reshape(ne, ns).astype(np.float32)
        out["nuclear_tables_aligned_to_primary_axis"] = True
    return out


def save_table_npz(path: str | Path, energy: dict, **meta: str) -> None:
    """Store an energy dict (arrays and scalars) in one compressed archive; string
    keyword arguments are kept beside it as metadata (`meta_<name>`)."""
    arrays = {}
    for k, v in energy.items():
        arrays[k] = np.asarray(v)
    for k, v in meta.items():
        arrays[f"meta_{k}"] = np.asarray(str(v))
    np.savez_compressed(path, **arrays)


def load_table_npz(path: str | Path) -> dict:
    """The energy dict stored by `save_table_npz` (metadata keys left out)."""
    z = np.load(path)
    out = {}
    for k in z.files:
        if k.startswith("meta_"):
            continue
        v = z[k]
        if v.ndim == 0:
            v = v.item()
            if isinstance(v, float) and k.startswith("n_"):
                v = int(v)
        out[k] = v
    return out


def _fmt(a) -> str:
    return " ".join(f"{float(x):.6g}" for x in np.asarray(a).reshape(-1))


def write_tables(tables_dir: str | Path, energy: dict) -> None:
    """Write an energy dict back in the reference's text formats."""
    d = Path(tables_dir)
    d.mkdir(parents=True, exist_ok=True)
    ne, ns = int(energy["n_energies"]), int(energy["n_energy_samples"])
    body = "\n".join([f"{ns} {ne}", "", _fmt(energy["energies_per_u"]), _fmt(energy["peak_depths"]),
                      _fmt(energy["scale_facts"]), _fmt(energy["cidd_matrix"])])
    (d / PROTON_FILE).write_text(body + "\n")
    for key, fname in (("density", DENSITY_FILE), ("sp", SP_FILE), ("rrl", RRL_FILE)):
        vec = energy[f"{key}_vector"]
        (d / fname).write_text(f"{len(vec)} {energy[f'{key}_scale_fact']:g}\n\n{_fmt(vec)}\n")
    if "nuc_weight_matrix" in energy:
        body = "\n".join([f"{ns} {ne}", "", _fmt(energy["energies_per_u"]), _fmt(energy["peak_depths"]),
                          _fmt(energy["scale_facts"]), _fmt(energy["nuc_weight_matrix"]),
                          _fmt(energy["nuc_sq_sigma_matrix"])])
        (d / NUCLEAR_FILE).write_text(body + "\n")


# ---- analytic models -----------------------------------------------------------

_ERF = np.vectorize(math.erf)


def _cidd_curve(range_mm: float, straggle_mm: float, z: np.ndarray, e0: float, p: float, alpha: float,
                fluence_loss_per_mm: float, tail: float) -> np.ndarray:
    """Cumulative integral depth dose (MeV per particle) on depths z (mm).

    Pristine energy loss from R = alpha * E^p, E0 - E_res(z), smeared by a
    Gaussian range straggling of width `straggle_mm` (the smearing of a cumulative
    curve is the cumulative of the smeared dose), weighted by a linear primary
    fluence loss, plus a fraction `tail` of fragment dose spread beyond the range."""
    fine = np.linspace(0.0, z[-1] + 6 * straggle_mm, 8192)
    resid = np.clip(range_mm - fine, 0.0, None)
    c0 = e0 - (resid / alpha) ** (1.0 / p)
    dz = fine[1] - fine[0]
    half = int(math.ceil(5 * straggle_mm / dz))
    t = np.arange(-half, half + 1) * dz
    kern = np.exp(-0.5 * (t / straggle_mm) ** 2)
    kern /= kern.sum()
    dose = np.gradient(c0, dz)
    dose = np.convolve(np.pad(dose, (half, half), mode="edge"), kern, mode="valid")
    dose *= np.clip(1.0 - fluence_loss_per_mm * fine, 0.0, None)
    if tail > 0.0:
        beyond = fine > range_mm
        dose[beyond] += tail * (e0 / range_mm) * np.exp(-(fine[beyond] - range_mm) / (0.3 * range_mm))
    c = np.concatenate([[0.0], np.cumsum(0.5 * (dose[1:] + dose[:-1]) * dz)])
    return np.interp(z, fine, c)


def _piecewise(x: np.ndarray, knots) -> np.ndarray:
    kx = np.array([k[0] for k in knots], dtype=np.float64)
    ky = np.array([k[1] for k in knots], dtype=np.float64)
    return np.interp(x, kx, ky)


def hu_luts() -> dict:
    """HU->density, HU->relative stopping power and density->radiation-length
    tables in the reference's layout (3072 samples, index = HU+1000 or density*1000)."""
    hu = np.arange(3072, dtype=np.float64) - 1000.0
    dens = _piecewise(hu, [(-1000, 0.0012), (-950, 0.044), (-120, 0.93), (-82, 0.95), (0, 1.0),
                           (60, 1.06), (200, 1.13), (1000, 1.60), (2071, 2.30)])
    sp = _piecewise(hu, [(-1000, 0.0011), (-950, 0.045), (-120, 0.94), (-82, 0.96), (0, 1.0),
                         (60, 1.05), (200, 1.10), (1000, 1.45), (2071, 1.85)])
    rho = np.arange(3072, dtype=np.float64) / 1000.0
    rrl = _piecewise(rho, [(0.0, 0.00273), (0.8, 0.00241), (1.0, 0.00259), (1.5, 0.00337), (3.07, 0.00450)])
    return {
        "n_density_samples": 3072, "density_scale_fact": 1.0, "density_vector": dens.astype(np.float32),
        "n_sp_samples": 3072, "sp_scale_fact": 1.0, "sp_vector": sp.astype(np.float32),
        "n_rrl_samples": 3072, "rrl_scale_fact": 1000.0, "rrl_vector": rrl.astype(np.float32),
    }


def _ion_tables(ranges_mm: np.ndarray, alpha: float, p: float, n_samples: int, peak_index: float,
                straggle_coef: float, straggle_pow: float, fluence_loss: float, tail: float,
                mev_scale: float) -> dict:
    energies = (ranges_mm / alpha) ** (1.0 / p)
    ne = ranges_mm.size
    cidd = np.zeros((ne, n_samples), dtype=np.float64)
    peaks = np.zeros(ne)
    scales = np.zeros(ne)
    for i, (r, e0) in enumerate(zip(ranges_mm, energies)):
        sigma = straggle_coef * (r / 10.0) ** straggle_pow * 10.0  # cm law, mm out
        # Bragg-peak depth of the smeared curve.
        zz = np.linspace(0.0, 1.3 * r, 4096)
        cc = _cidd_curve(r, sigma, zz, e0, p, alpha, fluence_loss, tail)
        peak = zz[int(np.argmax(np.gradient(cc, zz)))]
        scale = peak_index / peak
        depth = np.arange(n_samples, dtype=np.float64) / scale
        cidd[i] = _cidd_curve(r, sigma, depth, e0, p, alpha, fluence_loss, tail) * mev_scale
        peaks[i] = peak
        scales[i] = scale
    return {
        "n_energies": ne,
        "n_energy_samples": n_samples,
        "energies_per_u": energies.astype(np.float32),
        "peak_depths": peaks.astype(np.float32),
        "scale_facts": scales.astype(np.float32),
        "cidd_matrix": cidd.astype(np.float32),
    }


def synthetic_proton_tables(n_energies: int = 147, n_samples: int = 1024) -> dict:
    """Proton tables with the reference's axes: 147 energies of ~62-227 MeV and a
    1024-sample depth axis on which every Bragg peak sits at index 819."""
    ranges = np.linspace(31.0, 325.0, n_energies)
    t = _ion_tables(ranges, alpha=0.022, p=1.77, n_samples=n_samples, peak_index=819.0, straggle_coef=0.012,
                    straggle_pow=0.935, fluence_loss=0.0012, tail=0.0, mev_scale=1.602e-7)
    t.update(hu_luts())
    return t


def synthetic_carbon_tables(n_energies: int = 120, n_samples: int = 1024) -> dict:
    """Carbon-ion tables for 120-400 MeV/u in the same layout, with a fragment tail."""
    # Range in water of carbon ions, R = alpha * (E/u)^p with alpha/p fitted to
    # ~36 mm at 120 MeV/u and ~270 mm at 400 MeV/u.
    p = 1.675
    alpha = 270.0 / 400.0 ** p
    e = np.linspace(120.0, 400.0, n_energies)
    ranges = alpha * e ** p
    t = _ion_tables(ranges, alpha=alpha, p=p, n_samples=n_samples, peak_index=819.0, straggle_coef=0.004,
                    straggle_pow=0.935, fluence_loss=0.002, tail=0.08, mev_scale=1.602e-7)
    t.update(hu_luts())
    return t


def synthetic_nuclear_tables(energy: dict) -> dict:
    """Nuclear halo weight and squared-sigma tables aligned to `energy`'s axes
    (the layout of nuclear_weights_and_sigmas_fit.txt): the halo fraction grows
    with depth up to the peak and drops behind it; the halo variance (mm^2) grows
    with depth."""
    ne, ns = int(energy["n_energies"]), int(energy["n_energy_samples"])
    w = np.zeros((ne, ns), dtype=np.float64)
    s2 = np.zeros((ne, ns), dtype=np.float64)
    for i in range(ne):
        scale = float(energy["scale_facts"][i])
        peak = float(energy["peak_depths"][i])
        z = np.arange(ns) / scale
        frac = np.clip(z / max(peak, 1e-3), 0.0, 1.2)
        w[i] = 0.10 + 0.08 * np.minimum(frac, 1.0) - 0.04 * np.clip(frac - 1.0, 0.0, 0.2) / 0.2
        s2[i] = 40.0 + 90.0 * np.sin(0.5 * np.pi * np.minimum(frac, 1.0))
    out = dict(energy)
    out["nuc_weight_matrix"] = w.astype(np.float32)
    out["nuc_sq_sigma_matrix"] = s2.astype(np.float32)
    out["nuclear_tables_aligned_to_primary_axis"] = True
    return out
