"""Seeded synthetic workloads in the layout the reference's Python API takes.

No public dataset exists for this path; every input is generated from a seeded
numpy PCG64 stream:

* `water_phantom_case` - homogeneous water box along +z with one energy layer on
  an 11x11 square spot grid (the CPU-runnable plain-pipeline case).
* `heterogeneous_case` - body ellipsoid with Gaussian HU noise, a lung slab and
  two bone cylinders, one beam at gantry 90 deg with N energy layers of spots on a
  5 mm hexagonal grid over a spherical target (the headline 256x256x160 case and
  its scaled-down parity variants).

Each case is a dict with `ct` (float32 [Z][Y][X]), grid tuples (x, y, z order as
the reference's ct_dims/ct_resolution/ct_corner), the beam dict and the energy
dict of src/bindings/raytracedicom_pybind.cpp:1711-1847.
"""
from __future__ import annotations

import numpy as np

from .tables import synthetic_proton_tables

SEED_BASE = 20261203

_TABLE_CACHE: dict = {}


def proton_tables() -> dict:
    if "proton" not in _TABLE_CACHE:
        _TABLE_CACHE["proton"] = synthetic_proton_tables()
    return _TABLE_CACHE["proton"]


def subspot_lut(n_layers: int, n_side: int, sigma_mm: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    """[L][n_side^2][5] subspot table (dx, dy, weight, sigma_x, sigma_y): an
    n_side x n_side grid spanning +-1.5 sigma with Gaussian weights summing to 1."""
    out = np.zeros((n_layers, n_side * n_side, 5), dtype=np.float32)
    g = np.linspace(-1.5, 1.5, n_side)
    gx, gy = np.meshgrid(g, g, indexing="xy")
    w = np.exp(-0.5 * (gx ** 2 + gy ** 2)).reshape(-1)
    w /= w.sum()
    for layer in range(n_layers):
        s = float(sigma_mm[layer])
        out[layer, :, 0] = gx.reshape(-1) * s
        out[layer, :, 1] = gy.reshape(-1) * s
        out[layer, :, 2] = w
        out[layer, :, 3] = s / n_side
        out[layer, :, 4] = s / n_side
    return out


def _grid(dims, res):
    dims = tuple(int(d) for d in dims)
    res = tuple(float(r) for r in res)
    corner = tuple(-0.5 * (d - 1) * r for d, r in zip(dims, res))
    return dims, res, corner


def water_phantom_case(dims=(64, 64, 128), res=(2.0, 2.0, 2.0), energy_mev=150.0, n_side=11, spacing_mm=5.0,
                       sigma_mm=4.0, sad_mm=10000.0, ray_spacing=1.0, n_sub=7, seed=SEED_BASE + 1,
                       energy: dict | None = None) -> dict:
    """Homogeneous water: all HU = 0 passed as HU+1000 = 1000 (an all-zero HU volume
    would be auto-detected as density by the reference, raytracedicom_wrapper.cu:2333).
    `energy` is the table dict (default: the synthetic proton tables)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dims, res, corner = _grid(dims, res)
    ct = np.full((dims[2], dims[1], dims[0]), 1000.0, dtype=np.float32)
    g = (np.arange(n_side) - (n_side - 1) / 2.0) * spacing_mm
    px, py = np.meshgrid(g, g, indexing="xy")
    pos = np.stack([px.reshape(-1), py.reshape(-1)], axis=1).astype(np.float32)
    n = pos.shape[0]
    iso = np.zeros(3)
    bmz = np.array([0.0, 0.0, 1.0])
    beam = {
        "energies": np.array([energy_mev], dtype=np.float32),
        "spot_sigmas": np.array([[sigma_mm, sigma_mm]], dtype=np.float32),
        "ray_spacing": (ray_spacing, ray_spacing),
        "steps": 0,
        "source_dist": (sad_mm, sad_mm),
        "spot_offset": (0.0, 0.0, 0.0),
        "spot_delta": (spacing_mm, spacing_mm, 0.0),
        "beam_direction": tuple(bmz),
        "beam_xdir": (1.0, 0.0, 0.0),
        "beam_ydir": (0.0, 1.0, 0.0),
        "sad": sad_mm,
        "source_position": tuple(iso - bmz * sad_mm),
        "layer_spot_counts": np.array([n], dtype=np.int32),
        "spot_positions": pos.reshape(-1),
        "spot_weights": np.ones(n, dtype=np.float32),
        "subspot_data": subspot_lut(1, n_sub, np.array([sigma_mm]), rng),
    }
    return {"name": "water_phantom", "ct": ct, "ct_dims": dims, "ct_resolution": res, "ct_corner": corner,
            "dose_dims": dims, "dose_resolution": res, "dose_corner": corner, "beam": beam,
            "energy": proton_tables() if energy is None else energy}


def heterogeneous_ct(dims, res, rng: np.random.Generator) -> np.ndarray:
    """HU volume [Z][Y][X]: air -1000 outside a body ellipsoid (semi-axes 0.45 of
    the extents) of HU N(0, 20); a lung slab N(-800, 50) and two bone cylinders
    U(700, 1200) inside it."""
    nx, ny, nz = dims
    # Broadcast coordinates ([Z][1][1], [1][Y][1], [1][1][X]) keep the masks the
    # only full-size temporaries.
    z = np.arange(nz, dtype=np.float32)[:, None, None]
    y = np.arange(ny, dtype=np.float32)[None, :, None]
    x = np.arange(nx, dtype=np.float32)[None, None, :]
    cx, cy, cz = (nx - 1) / 2.0, (ny - 1) / 2.0, (nz - 1) / 2.0
    ax, ay, az = 0.45 * nx, 0.45 * ny, 0.45 * nz
    body = ((x - cx) / ax) ** 2 + ((y - cy) / ay) ** 2 + ((z - cz) / az) ** 2 <= 1.0
    ct = np.full((nz, ny, nx), -1000.0, dtype=np.float32)
    ct[body] = rng.normal(0.0, 20.0, size=int(body.sum())).astype(np.float32)
    # Lung slab: a band in y on the +y side of the body.
    lung = body & (y > cy + 0.10 * ny) & (y < cy + 0.30 * ny) & (np.abs(z - cz) < 0.30 * nz)
    ct[lung] = rng.normal(-800.0, 50.0, size=int(lung.sum())).astype(np.float32)
    # Two bone cylinders along z.
    for ox, oy in ((-0.18, -0.12), (0.20, -0.20)):
        r = 0.05 * min(nx, ny)
        cyl = body & (((x - (cx + ox * nx)) ** 2 + (y - (cy + oy * ny)) ** 2) <= r * r)
        ct[cyl] = rng.uniform(700.0, 1200.0, size=int(cyl.sum())).astype(np.float32)
    return ct


def hex_spots(radius_mm: float, pitch_mm: float) -> np.ndarray:
    """Hexagonal lattice points (rows pitch*sqrt(3)/2 apart, alternate rows shifted
    by pitch/2) inside a disc, [N][2] in mm."""
    dy = pitch_mm * np.sqrt(3.0) / 2.0
    pts = []
    nrow = int(np.ceil(radius_mm / dy)) + 1
    ncol = int(np.ceil(radius_mm / pitch_mm)) + 2
    for j in range(-nrow, nrow + 1):
        shift = 0.5 * pitch_mm if (j % 2) else 0.0
        for i in range(-ncol, ncol + 1):
            x, y = i * pitch_mm + shift, j * dy
            if x * x + y * y <= radius_mm * radius_mm:
                pts.append((x, y))
    return np.array(pts, dtype=np.float32)


def rotate_beam(beam: dict, gantry_deg: float) -> dict:
    """Copy of `beam` at another gantry angle (rotation about the z axis through the
    isocentre at the origin); 90 deg is the beam travelling along -x."""
    t = np.deg2rad(gantry_deg)
    d = np.array([-np.sin(t), -np.cos(t), 0.0])
    out = dict(beam)
    out["beam_direction"] = tuple(d)
    out["beam_xdir"] = (float(np.cos(t)), float(-np.sin(t)), 0.0)
    out["beam_ydir"] = (0.0, 0.0, 1.0)
    out["source_position"] = tuple(-d * float(beam["sad"]))
    return out


def legacy_beam(beam: dict) -> dict:
    """The beam without raw spot lists: its spots become the subspot table
    [L][maxSpots][5] = (x, y, w, sigma_x, sigma_y), which drives the legacy CPB
    fluence path (raytracedicom_wrapper.cu:3454-3507)."""
    counts = np.asarray(beam["layer_spot_counts"]).astype(int)
    pos = np.asarray(beam["spot_positions"], np.float32).reshape(-1, 2)
    w = np.asarray(beam["spot_weights"], np.float32)
    sig = np.asarray(beam["spot_sigmas"], np.float32).reshape(-1, 2)
    m = int(counts.max())
    sub = np.zeros((len(counts), m, 5), np.float32)
    off = 0
    for layer, c in enumerate(counts):
        sub[layer, :c, 0] = pos[off:off + c, 0]
        sub[layer, :c, 1] = pos[off:off + c, 1]
        sub[layer, :c, 2] = w[off:off + c]
        sub[layer, :c, 3] = sig[layer, 0]
        sub[layer, :c, 4] = sig[layer, 1]
        off += c
    out = {k: v for k, v in beam.items() if k not in ("layer_spot_counts", "spot_positions", "spot_weights")}
    out["subspot_data"] = sub
    return out


def to_centimetres(case: dict) -> dict:
    """The same case expressed in centimetres (CT z spacing < 0.3 switches the
    reference's length unit, raytracedicom_wrapper.cu:2729)."""
    out = dict(case)
    for k in ("ct_resolution", "ct_corner", "dose_resolution", "dose_corner"):
        out[k] = tuple(float(v) / 10.0 for v in case[k])
    b = dict(case["beam"])
    b["spot_positions"] = np.asarray(b["spot_positions"], np.float32) / 10.0
    b["spot_sigmas"] = np.asarray(b["spot_sigmas"], np.float32) / 10.0
    b["ray_spacing"] = tuple(float(v) / 10.0 for v in b["ray_spacing"])
    b["source_dist"] = tuple(float(v) / 10.0 for v in b["source_dist"])
    b["spot_delta"] = tuple(float(v) / 10.0 for v in b["spot_delta"])
    b["sad"] = float(b["sad"]) / 10.0
    b["source_position"] = tuple(float(v) / 10.0 for v in b["source_position"])
    sub = np.asarray(b["subspot_data"], np.float32).copy()
    sub[..., [0, 1, 3, 4]] /= 10.0
    b["subspot_data"] = sub
    out["beam"] = b
    return out


def with_spot_directions(beam: dict, sad_x: float, sad_y: float) -> dict:
    """Adds per-spot beam directions diverging from virtual sources at sad_x / sad_y
    (the CarbonPBS beam_dir input from which the reference recovers the source
    distances, raytracedicom_wrapper.cu:1847-1921)."""
    bz = np.asarray(beam["beam_direction"], np.float64)
    bx = np.asarray(beam["beam_xdir"], np.float64)
    by = np.asarray(beam["beam_ydir"], np.float64)
    pos = np.asarray(beam["spot_positions"], np.float64).reshape(-1, 2)
    d = bz[None, :] + bx[None, :] * (pos[:, :1] / sad_x) + by[None, :] * (pos[:, 1:] / sad_y)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    out = dict(beam)
    out["spot_beam_directions"] = d.astype(np.float32).reshape(-1)
    return out


def heterogeneous_case(dims=(256, 256, 160), res=(2.0, 2.0, 2.0), n_layers=20, e_range=(70.0, 180.0),
                       target_radius_mm=32.0, hex_pitch_mm=5.0, sigma_range=(6.0, 3.0), sad_mm=2000.0,
                       ray_spacing=1.0, n_sub=7, seed=SEED_BASE + 2, energy: dict | None = None) -> dict:
    """The heterogeneous phantom and its hexagonal-grid beam; `energy` is the table
    dict (default: the synthetic proton tables)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dims, res, corner = _grid(dims, res)
    ct = heterogeneous_ct(dims, res, rng)
    energies = np.linspace(e_range[0], e_range[1], n_layers).astype(np.float32)
    sig = np.linspace(sigma_range[0], sigma_range[1], n_layers).astype(np.float32)
    spots = hex_spots(target_radius_mm, hex_pitch_mm)
    counts = np.full(n_layers, spots.shape[0], dtype=np.int32)
    pos = np.tile(spots, (n_layers, 1))
    weights = rng.lognormal(0.0, 0.5, size=pos.shape[0]).astype(np.float32)
    iso = np.zeros(3)
    bmz = np.array([-1.0, 0.0, 0.0])  # gantry 90 deg: the beam travels along -x
    beam = {
        "energies": energies,
        "spot_sigmas": np.stack([sig, sig], axis=1),
        "ray_spacing": (ray_spacing, ray_spacing),
        "steps": 0,
        "source_dist": (sad_mm, sad_mm),
        "spot_offset": (0.0, 0.0, 0.0),
        "spot_delta": (hex_pitch_mm, hex_pitch_mm * np.sqrt(3.0) / 2.0, 0.0),
        "beam_direction": tuple(bmz),
        "beam_xdir": (0.0, 1.0, 0.0),
        "beam_ydir": (0.0, 0.0, 1.0),
        "sad": sad_mm,
        "source_position": tuple(iso - bmz * sad_mm),
        "layer_spot_counts": counts,
        "spot_positions": pos.reshape(-1),
        "spot_weights": weights,
        "subspot_data": subspot_lut(n_layers, n_sub, sig, rng),
    }
    return {"name": "heterogeneous", "ct": ct, "ct_dims": dims, "ct_resolution": res, "ct_corner": corner,
            "dose_dims": dims, "dose_resolution": res, "dose_corner": corner, "beam": beam,
            "energy": proton_tables() if energy is None else energy}


def inverse_planning_case(dims=(64, 64, 128), res=(2.0, 2.0, 2.0), n_beams=4, n_layers=36, e_range=(66.0, 112.0),
                          field_mm=70.0, pitch_mm=5.0, sigma_mm=4.0, target_radius_mm=25.0, shell_mm=20.0,
                          prescription_gy=2.0, sad_mm=10000.0, ray_spacing=1.0, n_sub=7,
                          seed=SEED_BASE + 4, energy: dict | None = None) -> dict:
    """Inverse-planning workload: the water box of `water_phantom_case`, `n_beams`
    coplanar beams (gantry 0, 360/n, ...), each with `n_layers` energy layers of a
    square spot grid over the field (36 x 225 = 8100 spots per beam by default) and
    lognormal weights; a target sphere of `target_radius_mm` at the isocentre with a
    `prescription_gy` prescription and a surrounding `shell_mm` shell with 0 Gy.
    Adds `beams`, `target` and `shell` (bool [Z][Y][X]) and `prescription`."""
    rng = np.random.Generator(np.random.PCG64(seed))
    base = water_phantom_case(dims=dims, res=res, sigma_mm=sigma_mm, sad_mm=sad_mm, ray_spacing=ray_spacing,
                              n_sub=n_sub, seed=seed, energy=energy)
    n_side = int(round(field_mm / pitch_mm)) + 1
    g = (np.arange(n_side) - (n_side - 1) / 2.0) * pitch_mm
    px, py = np.meshgrid(g, g, indexing="xy")
    spots = np.stack([px.reshape(-1), py.reshape(-1)], axis=1).astype(np.float32)
    energies = np.linspace(e_range[0], e_range[1], n_layers).astype(np.float32)
    counts = np.full(n_layers, spots.shape[0], dtype=np.int32)
    beam = dict(base["beam"])
    beam.update({
        "energies": energies,
        "spot_sigmas": np.tile(np.array([[sigma_mm, sigma_mm]], np.float32), (n_layers, 1)),
        "spot_delta": (pitch_mm, pitch_mm, 0.0),
        "layer_spot_counts": counts,
        "spot_positions": np.tile(spots, (n_layers, 1)).reshape(-1),
        "subspot_data": subspot_lut(n_layers, n_sub, np.full(n_layers, sigma_mm), rng),
    })
    beams = []
    for k in range(n_beams):
        b = rotate_beam(beam, 360.0 * k / n_beams)
        b["spot_weights"] = rng.lognormal(0.0, 0.5, size=int(counts.sum())).astype(np.float32)
        beams.append(b)
    dims_, res_, corner = _grid(dims, res)
    z, y, x = np.meshgrid(*(corner[i] + res_[i] * np.arange(dims_[i]) for i in (2, 1, 0)), indexing="ij")
    r = np.sqrt(x * x + y * y + z * z)
    out = dict(base)
    out.update({"name": "inverse_planning", "beam": beams[0], "beams": beams, "target": r <= target_radius_mm,
                "shell": (r > target_radius_mm) & (r <= target_radius_mm + shell_mm),
                "prescription": float(prescription_gy)})
    return out


# ---- serving stream (mixed CT sizes, beams, spot counts and ions) -------------

SERVING_CT_CLASSES = (((128, 128, 128), (2.0, 2.0, 2.0)),
                      ((256, 256, 160), (2.0, 2.0, 2.0)),
                      ((512, 512, 200), (1.0, 1.0, 1.0)))


def carbon_tables() -> dict:
    """Synthetic carbon-ion tables (120-400 MeV/u) with their nuclear halo tables."""
    from .tables import synthetic_carbon_tables, synthetic_nuclear_tables

    if "carbon" not in _TABLE_CACHE:
        _TABLE_CACHE["carbon"] = synthetic_nuclear_tables(synthetic_carbon_tables())
    return _TABLE_CACHE["carbon"]


def heavy_tailed_spots(rng: np.random.Generator, lo: int = 500, hi: int = 20000, alpha: float = 1.1) -> int:
    """Pareto(alpha) spot count with minimum `lo`, clipped at `hi`."""
    return int(min(hi, np.floor(lo * (1.0 - rng.uniform()) ** (-1.0 / alpha))))


def field_beam(n_spots: int, ion: str, gantry_deg: float, rng: np.random.Generator, pitch_mm: float = 5.0,
               sad_mm: float = 2000.0, ray_spacing: float = 1.0, n_sub: int = 7) -> dict:
    """A coplanar field of about `n_spots` spots: n_spots/250 energy layers (4 to
    40) of a hexagonal spot disc, proton 70-180 MeV (sigma 6 -> 3 mm) or carbon
    120-400 MeV/u (sigma 4 -> 2 mm); unit weights (a request sets its own)."""
    n_layers = int(np.clip(round(n_spots / 250.0), 4, 40))
    per_layer = max(n_spots // n_layers, 7)
    radius = float(np.sqrt(per_layer * pitch_mm * pitch_mm * np.sqrt(3.0) / 2.0 / np.pi))
    spots = hex_spots(radius, pitch_mm)
    e_range, s_range = ((70.0, 180.0), (6.0, 3.0)) if ion == "proton" else ((120.0, 400.0), (4.0, 2.0))
    energies = np.linspace(e_range[0], e_range[1], n_layers).astype(np.float32)
    sig = np.linspace(s_range[0], s_range[1], n_layers).astype(np.float32)
    counts = np.full(n_layers, spots.shape[0], dtype=np.int32)
    bmz = np.array([-1.0, 0.0, 0.0])
    beam = {
        "energies": energies,
        "spot_sigmas": np.stack([sig, sig], axis=1),
        "ray_spacing": (ray_spacing, ray_spacing),
        "steps": 0,
        "source_dist": (sad_mm, sad_mm),
        "spot_offset": (0.0, 0.0, 0.0),
        "spot_delta": (pitch_mm, pitch_mm * np.sqrt(3.0) / 2.0, 0.0),
        "beam_direction": tuple(bmz),
        "beam_xdir": (0.0, 1.0, 0.0),
        "beam_ydir": (0.0, 0.0, 1.0),
        "sad": sad_mm,
        "source_position": tuple(-bmz * sad_mm),
        "layer_spot_counts": counts,
        "spot_positions": np.tile(spots, (n_layers, 1)).reshape(-1),
        "spot_weights": np.ones(int(counts.sum()), np.float32),
        "subspot_data": subspot_lut(n_layers, n_sub, sig, rng),
    }
    return rotate_beam(beam, gantry_deg)


def serving_workload(n_requests: int = 1000, rate_hz: float = 100.0, patients_per_class: int = 4,
                     fields_per_patient: int = 4, carbon_fraction: float = 0.2, seed: int = SEED_BASE + 5,
                     ct_classes=SERVING_CT_CLASSES, max_spots: int = 20000,
                     proton_energy: dict | None = None) -> dict:
    """Seeded stream of dose requests: patients with CTs uniform among the three
    size classes of SERVING_CT_CLASSES (heterogeneous_ct recipe), each with
    `fields_per_patient` coplanar fields of a heavy-tailed spot count (500-20000)
    in a proton and a carbon variant; requests arrive as a Poisson process of
    `rate_hz`, pick a patient uniformly, 1-4 of its fields and an ion (carbon with
    `carbon_fraction`, with the nuclear halo). Spot weights are drawn per request
    (`request_beams`). `proton_energy` is the proton table dict (default: the
    synthetic proton tables); carbon uses the synthetic carbon tables."""
    rng = np.random.Generator(np.random.PCG64(seed))
    patients = []
    for c, (dims, res) in enumerate(ct_classes):
        for k in range(patients_per_class):
            pid = len(patients)
            prng = np.random.Generator(np.random.PCG64(seed + 1000 + pid))
            dims_, res_, corner = _grid(dims, res)
            gantries = (rng.uniform(0.0, 360.0) + 360.0 / fields_per_patient * np.arange(fields_per_patient)) % 360.0
            fields = []
            for g in gantries:
                n = heavy_tailed_spots(rng, hi=max_spots)
                fields.append({"spots": n, "gantry": float(g),
                               "proton": field_beam(n, "proton", float(g), prng),
                               "carbon": field_beam(n, "carbon", float(g), prng)})
            patients.append({"id": pid, "size_class": c, "ct": heterogeneous_ct(dims_, res_, prng),
                             "ct_dims": dims_, "ct_resolution": res_, "ct_corner": corner, "dose_dims": dims_,
                             "dose_resolution": res_, "dose_corner": corner, "fields": fields})
    gaps = rng.exponential(1.0 / rate_hz, size=n_requests)
    arrivals = np.cumsum(gaps) - gaps[0]
    requests = []
    for i in range(n_requests):
        pid = int(rng.integers(len(patients)))
        nb = int(rng.integers(1, 5))
        nb = min(nb, fields_per_patient)
        fids = sorted(int(f) for f in rng.choice(fields_per_patient, nb, replace=False))
        ion = "carbon" if rng.uniform() < carbon_fraction else "proton"
        requests.append({"index": i, "arrival_s": float(arrivals[i]), "patient": pid, "fields": fids, "ion": ion,
                         "seed": seed + 100000 + i})
    return {"patients": patients, "requests": requests, "rate_hz": rate_hz,
            "energy": {"proton": proton_tables() if proton_energy is None else proton_energy,
                       "carbon": carbon_tables()}}


def request_beams(workload: dict, req: dict) -> list:
    """The request's beams with their lognormal(0, 0.5) spot weights."""
    rng = np.random.Generator(np.random.PCG64(req["seed"]))
    p = workload["patients"][req["patient"]]
    out = []
    for f in req["fields"]:
        b = dict(p["fields"][f][req["ion"]])
        b["spot_weights"] = rng.lognormal(0.0, 0.5, size=b["spot_weights"].size).astype(np.float32)
        out.append(b)
    return out


# ---- water-equivalence import (CarbonPBS rayweq) -------------------------------

def weq_volume(n_xy: int, pitch_mm: float, n_steps: int, step_mm: float, rng: np.random.Generator) -> tuple:
    """Synthetic exporter depths in beam's-eye coordinates: per lateral texel (u, v)
    (pitch_mm apart, centred on the beam axis) and depth t = (k + 1) * step_mm from
    the start plane, relative stopping power 0 in air before a curved skin surface
    t_in = 30 mm + (u^2 + v^2) / 500 mm, 1.0 +- 1 % in tissue, 0.25 in a lung band
    (v > 8 mm, 20 mm to 50 mm past the skin) and 1.7 in a bone slab (|u - 6| < 5 mm,
    35 mm to 45 mm past the skin); the depth is the running sum of rsp * step_mm.
    Returns (weq [nx][ny][steps] float32, lateral origin mm)."""
    x0 = -0.5 * (n_xy - 1) * pitch_mm
    u = (x0 + pitch_mm * np.arange(n_xy))[:, None, None]
    v = (x0 + pitch_mm * np.arange(n_xy))[None, :, None]
    t = ((np.arange(n_steps) + 1) * step_mm)[None, None, :]
    t_in = 30.0 + (u * u + v * v) / 500.0
    past = t - t_in
    rsp = np.where(past >= 0.0, 1.0 + 0.01 * rng.standard_normal((n_xy, n_xy, 1)), 0.0)
    rsp = np.where((v > 8.0) & (past >= 20.0) & (past < 50.0), 0.25, rsp)
    rsp = np.where((np.abs(u - 6.0) < 5.0) & (past >= 35.0) & (past < 45.0), 1.7, rsp)
    weq = np.cumsum(rsp * step_mm, axis=2).astype(np.float32)
    return weq, float(x0)


def weq_case(dims=(64, 64, 48), res=(2.0, 2.0, 2.0), n_layers=3, e_range=(80.0, 120.0), target_radius_mm=14.0,
             hex_pitch_mm=5.0, sigma_range=(6.0, 3.0), sad_mm=2000.0, ray_mm=1.0, n_sub=7, index_positions=True,
             seed=SEED_BASE + 6) -> dict:
    """A beam driven by an imported water-equivalence volume (the CarbonPBS rayweq
    contract): the heterogeneous_case CT fixes the dose grid and the beam geometry,
    and `water_equivalence` = the 9-value header [depth0, step, nSteps, y0, dy, ny,
    x0, dx, nx] followed by weq_volume's depths. The header's depth origin and step
    are the CT plan's start plane and step, so the BEV start plane stays where the CT
    would put it. With index_positions the spot positions are rayweq texel
    coordinates (texel i centred at i + 0.5), as CarbonPBS exports them."""
    from .cudaCalDoseRTD import plan_beam

    rng = np.random.Generator(np.random.PCG64(seed))
    case = heterogeneous_case(dims=dims, res=res, n_layers=n_layers, e_range=e_range,
                              target_radius_mm=target_radius_mm, hex_pitch_mm=hex_pitch_mm, sigma_range=sigma_range,
                              sad_mm=sad_mm, ray_spacing=ray_mm, n_sub=n_sub, seed=seed)
    beam = dict(case["beam"])
    st = plan_beam(beam, case["energy"], case["ct_dims"], case["ct_resolution"], case["ct_corner"],
                   case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    step = abs(float(st["fan_delta"][2]))
    n_steps = int(st["tracer_steps"])
    depth0 = 0.5 * (float(st["source_dist"][0]) + float(st["source_dist"][1])) - float(st["fan_corner"][2])
    half = target_radius_mm + 3.0 * max(sigma_range) + 8.0
    n_xy = 2 * int(np.ceil(half / ray_mm)) + 1
    weq, x0 = weq_volume(n_xy, ray_mm, n_steps, step, rng)
    header = np.array([depth0, step, n_steps, x0, ray_mm, n_xy, x0, ray_mm, n_xy], np.float32)
    beam["water_equivalence"] = np.concatenate([header, weq.reshape(-1)])
    beam["ray_weq_header"] = header
    if index_positions:
        pos = np.asarray(beam["spot_positions"], np.float32).reshape(-1, 2)
        beam["spot_positions"] = ((pos - np.array([x0, x0], np.float32)) / ray_mm + 0.5).astype(np.float32).reshape(-1)
        beam["spot_positions_are_indices"] = True
    out = dict(case)
    out.update({"name": "weq", "beam": beam, "weq": weq})
    return out


def carbonpbs_export(case: dict, idd_step_mm: float = 1.0, idd_samples: int = 400) -> dict:
    """The arguments of a cuFinalDose call (the CarbonPBS export) for a weq_case
    beam: the rayweq array, spot texel coordinates, weights and layer counts, per-
    spot directions, the subspot table with the spot sigma in its sigma columns, and
    an IDD table on one common depth axis (idd_step_mm spacing) taken from the
    case's CIDD tables (the derivative of each energy's CIDD curve, resampled)."""
    b = case["beam"]
    e = case["energy"]
    ne, ns = int(e["n_energies"]), int(e["n_energy_samples"])
    cidd = np.asarray(e["cidd_matrix"], np.float64).reshape(ne, ns)
    z = np.arange(idd_samples + 1) * idd_step_mm
    idd = np.zeros((ne, idd_samples), np.float32)
    for i in range(ne):
        c = np.interp(z * float(e["scale_facts"][i]), np.arange(ns), cidd[i])
        idd[i] = (np.diff(c) / idd_step_mm).astype(np.float32)
    n = int(np.sum(b["layer_spot_counts"]))
    d = np.asarray(b["beam_direction"], np.float32)
    dims = case["dose_dims"]
    # The contract reads each layer's spot sigma from its first subspot row
    # (raytracedicom_pybind.cpp:640-657): the subspots carry the spot sigma.
    sub = np.asarray(b["subspot_data"], np.float32).copy()
    sub[:, :, 3:5] = np.asarray(b["spot_sigmas"], np.float32).reshape(-1, 1, 2)
    return {
        "rayweq": np.asarray(b["water_equivalence"], np.float32),
        "roiIdx": np.zeros(0, np.int32),
        "all_energies": np.repeat(np.asarray(b["energies"], np.float32), np.asarray(b["layer_spot_counts"])),
        "sourcePos": np.asarray(b["source_position"], np.float32).reshape(3, 1),
        "tmpBeamDir": np.tile(d, (n, 1)),
        "bmxdir": np.asarray(b["beam_xdir"], np.float32),
        "bmydir": np.asarray(b["beam_ydir"], np.float32),
        "corner": np.asarray(case["dose_corner"], np.float32),
        "resolution": np.asarray(case["dose_resolution"], np.float32),
        "dims": np.asarray(dims, np.int32),
        "longitudalCutoff": None,
        "enelist": np.asarray(e["energies_per_u"], np.float32),
        "idddata": idd,
        "iddsetting": np.array([0.0, idd_step_mm, idd_samples], np.float32),
        "profiledata": None,
        "profilesetting": None,
        "beamparadata": None,
        "subspotdata": sub,
        "layerInfo": np.asarray(b["layer_spot_counts"], np.int32),
        "layerEnergy": np.asarray(b["energies"], np.float32),
        "idbeamxy": np.asarray(b["spot_positions"], np.float32).reshape(-1, 2),
        "nPar": np.asarray(b["spot_weights"], np.float32),
        "sad": float(b["sad"]),
    }


def carbon_case(dims=(512, 512, 200), res=(1.0, 1.0, 1.0), gantries=(0.0, 120.0, 240.0), n_layers=40,
                e_range=(120.0, 400.0), spots_per_layer=125, pitch_mm=5.0, sigma_range=(4.0, 2.0), sad_mm=2000.0,
                ray_spacing=1.0, n_sub=9, seed=SEED_BASE + 3) -> dict:
    """Carbon-ion plan with the nuclear halo: the heterogeneous_ct recipe on
    `dims` at `res`, one beam per gantry angle, `n_layers` layers spanning
    `e_range` MeV/u with about `spots_per_layer` spots each on a hexagonal grid,
    lognormal(0, 0.5) weights, sigma falling linearly over `sigma_range`,
    n_sub x n_sub subspots, and the synthetic carbon tables with their nuclear
    halo tables (carbon_tables)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dims_, res_, corner = _grid(dims, res)
    ct = heterogeneous_ct(dims_, res_, rng)
    radius = float(np.sqrt(spots_per_layer * pitch_mm * pitch_mm * np.sqrt(3.0) / 2.0 / np.pi))
    spots = hex_spots(radius, pitch_mm)
    energies = np.linspace(e_range[0], e_range[1], n_layers).astype(np.float32)
    sig = np.linspace(sigma_range[0], sigma_range[1], n_layers).astype(np.float32)
    counts = np.full(n_layers, spots.shape[0], dtype=np.int32)
    bmz = np.array([-1.0, 0.0, 0.0])
    base = {
        "energies": energies,
        "spot_sigmas": np.stack([sig, sig], axis=1),
        "ray_spacing": (ray_spacing, ray_spacing),
        "steps": 0,
        "source_dist": (sad_mm, sad_mm),
        "spot_offset": (0.0, 0.0, 0.0),
        "spot_delta": (pitch_mm, pitch_mm * np.sqrt(3.0) / 2.0, 0.0),
        "beam_direction": tuple(bmz),
        "beam_xdir": (0.0, 1.0, 0.0),
        "beam_ydir": (0.0, 0.0, 1.0),
        "sad": sad_mm,
        "source_position": tuple(-bmz * sad_mm),
        "layer_spot_counts": counts,
        "spot_positions": np.tile(spots, (n_layers, 1)).reshape(-1),
        "subspot_data": subspot_lut(n_layers, n_sub, sig, rng),
    }
    beams = []
    for g in gantries:
        b = rotate_beam(base, float(g))
        b["spot_weights"] = rng.lognormal(0.0, 0.5, size=int(counts.sum())).astype(np.float32)
        beams.append(b)
    return {"name": "carbon", "ct": ct, "ct_dims": dims_, "ct_resolution": res_, "ct_corner": corner,
            "dose_dims": dims_, "dose_resolution": res_, "dose_corner": corner, "beam": beams[0], "beams": beams,
            "energy": carbon_tables()}


def with_carbon_profile(beam: dict, n_gauss: int = 2, depth_n: int = 96, depth_step_mm: float = 2.0,
                        rows: str = "layers", seed: int = SEED_BASE + 7) -> dict:
    """The beam with a seeded CarbonPBS lateral profile model in the layout of the
    reference's RTDBeamSettings (raytracedicom_integration.h:71-76):
    profile_data [rows][depth_n][2 n_gauss + 1] (n_gauss weights, n_gauss sigmas in
    mm, one overall weight), profile_setting [depth0, step, depth_n], beam_para_data
    [rows][3] = (2 sigmaIso^2, rtheta, theta^2) and beam_para_pos. `rows` = "layers"
    gives one row per energy layer; "energies" gives rows on a separate energy axis
    (profile_energies) of 1.5x as many rows spanning the layers' energies, and no
    beam-parameter rows of that count (the reference then reads the rows from the
    energy axis)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    energies = np.asarray(beam["energies"], np.float32)
    L = energies.size
    if rows == "energies":
        n_rows = max(2, int(round(1.5 * L)))
        axis = np.linspace(float(energies.min()) - 2.0, float(energies.max()) + 2.0, n_rows).astype(np.float32)
    else:
        n_rows = L
        axis = None
    d = np.arange(depth_n, dtype=np.float64) * depth_step_mm
    ch = 2 * n_gauss + 1
    prof = np.zeros((n_rows, depth_n, ch), np.float64)
    for r in range(n_rows):
        w = rng.uniform(0.5, 1.0, n_gauss)
        w[1:] *= 0.3
        for g in range(n_gauss):
            prof[r, :, g] = w[g] * (1.0 + 0.1 * np.sin(d / (40.0 + 10.0 * g)))
            prof[r, :, n_gauss + g] = (1.2 + 2.5 * g) * (1.0 + d / 300.0) + rng.uniform(0.0, 0.3)
        prof[r, :, ch - 1] = np.clip(1.0 - 0.25 * d / d[-1] + rng.uniform(-0.02, 0.02), 0.0, None)
    sig_iso = np.linspace(4.0, 3.0, L if axis is None else L + 1)
    para = np.stack([2.0 * sig_iso ** 2, np.full_like(sig_iso, 0.002), np.full_like(sig_iso, 2.5e-5)], axis=1)
    out = dict(beam)
    out["profile_data"] = prof.astype(np.float32).reshape(-1)
    out["profile_setting"] = np.array([0.0, depth_step_mm, depth_n], np.float32)
    out["beam_para_data"] = para.astype(np.float32).reshape(-1)
    out["beam_para_pos"] = float(beam.get("sad", 0.0)) * 0.0
    if axis is not None:
        out["profile_energies"] = axis
    return out


def bio_model(model: str = "lq", energies=(60.0, 240.0), n_rows: int = 12, depth_step_mm: float = 0.5,
              max_depth_mm: float = 320.0) -> dict:
    """A seeded-free analytic biological model in the layout of PbsBioModel: a LET
    table (keV/um) that rises from an entrance plateau towards each energy's range
    (Bragg-Kleeman, R = 0.022 E^1.77 mm) and falls off behind it, and LQ alpha /
    beta (or MKM z1D) tables on a log10(LET) axis of 0.01 steps (the reference's
    lqData indexing, carbonPBS/deviceCalDose.cu:694-695). Synthetic: the reference
    ships no LET or LQ tables."""
    e = np.linspace(energies[0], energies[1], n_rows)
    depth = np.arange(0.0, max_depth_mm, depth_step_mm)
    let = np.zeros((n_rows, depth.size))
    for i, en in enumerate(e):
        r = 0.022 * en ** 1.77
        resid = np.clip(r - depth, 0.3, None)
        let[i] = np.where(depth <= r + 2.0, 0.4 + 12.0 / np.sqrt(resid + 0.5), 0.5)
    logl = np.arange(0.0, 3.0, 0.01)
    L = 10.0 ** logl
    out = {"model": model, "let_table": let.astype(np.float32), "let_energies": e.astype(np.float32),
           "let_depth0": 0.0, "let_depth_step": depth_step_mm, "let_samples": 5, "est_dimension": 2.0,
           "range_shifter": 0.0, "lq_log0": 0.0, "lq_log_step": 0.01}
    if model == "lq":
        # RBE near 1 at low LET: alpha 0.33 / Gy, beta 0.06 / Gy^2 give the reference's
        # 10 % survival photon dose of 3.99 Gy (LQRBEKernel's constant).
        out["lq_alpha"] = (0.33 + 0.05 * L / (1.0 + L / 150.0)).astype(np.float32)
        out["lq_beta"] = (0.06 * np.ones_like(L) / (1.0 + L / 500.0)).astype(np.float32)
    else:
        # MKM's photon reference of mkmRBEMapKernel (alphar, betar = 0.3312, 0.0593).
        out["z1d"] = (0.2 * L / (1.0 + L / 80.0)).astype(np.float32)
        out["alpha0"], out["beta0"] = 0.3312, 0.0593
    return out
