"""ctypes wrapper of the CPU oracle (test infrastructure only).

Only the tests, `__graft_entry__.smoke()` and bench.py's CPU-baseline leg use this
module, as the checker of the CUDA library. It builds liboracle.so with the
Makefile beside it when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_FP = C.POINTER(C.c_float)
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
_UP = C.POINTER(C.c_ubyte)


class OraclePlan(C.Structure):
    _fields_ = [
        ("num_layers", C.c_int), ("conv_mode", C.c_int),
        ("ray_x", C.c_int), ("ray_y", C.c_int), ("pitch_x", C.c_int), ("pitch_y", C.c_int),
        ("tiles_x", C.c_int), ("tiles_y", C.c_int), ("steps", C.c_int),
        ("lat_nx", C.c_int), ("lat_ny", C.c_int),
        ("lat_dx", C.c_float), ("lat_dy", C.c_float), ("lat_ox", C.c_float), ("lat_oy", C.c_float),
        ("cpb_corner", C.c_float * 2), ("cpb_res", C.c_float * 2),
        ("fan_corner", C.c_float * 3), ("fan_delta", C.c_float * 3),
        ("source_dist", C.c_float * 2),
        ("len_to_mm", C.c_float), ("energy_depth_to_mm", C.c_float), ("max_peak_depth_mm", C.c_float),
        ("bev_x", C.c_int), ("bev_y", C.c_int),
        ("nuc_x", C.c_int), ("nuc_y", C.c_int), ("nuc_bev_x", C.c_int), ("nuc_bev_y", C.c_int),
    ]


class OracleCapture(C.Structure):
    _fields_ = [
        ("density", _DP), ("wepl", _DP), ("first_inside", _IP), ("first_outside", _IP), ("wepl_min", _DP),
        ("beam_ints", _IP), ("ray_weights", _DP), ("entry_sigma", _FP), ("idd", _DP), ("rsigma", _DP),
        ("codes", _UP), ("layer_ints", _IP), ("layer_box", _IP), ("hist", _IP), ("batched", _IP),
        ("bev", _DP), ("superpose_fma", C.c_double),
        ("nuc_idd", _DP), ("nuc_rsigma", _DP), ("nuc_codes", _UP), ("nuc_hist", _IP), ("nuc_batched", _IP),
        ("nuc_bev", _DP), ("ray_to_nuc", _IP), ("nuc_superpose_fma", C.c_double),
    ]


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    from subsecondpbs_b200 import _lib as P

    lib = C.CDLL(str(LIB))
    lib.oracle_plan.restype = C.c_int
    lib.oracle_plan.argtypes = [C.POINTER(P.PbsBeamDesc), C.POINTER(P.PbsEnergyDesc), _IP, _FP, _FP, _IP, _FP, _FP,
                                C.POINTER(OraclePlan), _FP, _FP, C.c_size_t]
    lib.oracle_dose.restype = C.c_int
    lib.oracle_dose.argtypes = [_FP, _IP, _FP, _FP, _DP, _IP, _FP, _FP, C.POINTER(P.PbsBeamDesc), C.c_size_t,
                                C.POINTER(P.PbsEnergyDesc), C.c_int, C.c_int, C.c_int, C.POINTER(OracleCapture)]
    lib.oracle_dose_nuclear.restype = C.c_int
    lib.oracle_dose_nuclear.argtypes = [_FP, _IP, _FP, _FP, _DP, _IP, _FP, _FP, C.POINTER(P.PbsBeamDesc),
                                        C.c_size_t, C.POINTER(P.PbsEnergyDesc), C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.POINTER(OracleCapture)]
    lib.oracle_radius_bucket.restype = C.c_int
    lib.oracle_radius_bucket.argtypes = [C.c_float]
    lib.oracle_batch.restype = None
    lib.oracle_batch.argtypes = [_IP, _IP, _IP]
    lib.oracle_last_error.restype = C.c_char_p
    lib.oracle_set_carbon_profile.restype = None
    lib.oracle_set_carbon_profile.argtypes = [C.c_int]
    lib.oracle_set_bio.restype = None
    lib.oracle_set_bio.argtypes = [C.POINTER(P.PbsBioModel), _DP]
    lib.oracle_bio_map.restype = None
    lib.oracle_bio_map.argtypes = [C.POINTER(P.PbsBioModel), _DP, C.c_size_t, C.c_int, _DP]
    _lib = lib
    return lib


def _err(rc):
    if rc != 0:
        raise RuntimeError(f"oracle status {rc}: {load().oracle_last_error().decode()}")


def plan(case: dict, beam: dict | None = None, with_lattice: bool = False) -> dict:
    from subsecondpbs_b200 import _lib as P
    from subsecondpbs_b200.cudaCalDoseRTD import _with_luts

    lib = load()
    beam = beam if beam is not None else case["beam"]
    bd, kb = P.beam_desc(beam)
    ed, ke = P.energy_desc(_with_luts(case["energy"], None))
    op = OraclePlan()
    n_layers = len(np.asarray(beam["energies"]).reshape(-1))
    lp = np.zeros((n_layers, 8), dtype=np.float32)
    _err(lib.oracle_plan(C.byref(bd), C.byref(ed), P.int3(case["ct_dims"]), P.float3(case["ct_resolution"]),
                         P.float3(case["ct_corner"]), P.int3(case["dose_dims"]), P.float3(case["dose_resolution"]),
                         P.float3(case["dose_corner"]), C.byref(op), lp.ctypes.data_as(_FP), None, 0))
    out = {name: (list(getattr(op, name)) if isinstance(getattr(op, name), C.Array) else getattr(op, name))
           for name, _ in OraclePlan._fields_}
    out["layer_params"] = lp
    if with_lattice and op.conv_mode == 0:
        lat = np.zeros((n_layers, op.lat_ny, op.lat_nx), dtype=np.float32)
        _err(lib.oracle_plan(C.byref(bd), C.byref(ed), P.int3(case["ct_dims"]), P.float3(case["ct_resolution"]),
                             P.float3(case["ct_corner"]), P.int3(case["dose_dims"]),
                             P.float3(case["dose_resolution"]), P.float3(case["dose_corner"]), C.byref(op), None,
                             lat.ctypes.data_as(_FP), lat.size))
        out["lattice"] = lat
    del kb, ke
    return out


def dose(case: dict, beams: list | None = None, initial=None, ct_type: int = 0, compat_bev_z_shift: bool = False,
         threads: int = 0, capture: bool = False, capture_layers: bool = False, nuclear_model: int = -1,
         carbon_profile: int = 0, bio: dict | None = None) -> dict:
    """Run the oracle; returns {'dose': float64 [Z][Y][X], 'capture': {...}}.
    `nuclear_model` -1 runs without the nuclear halo; 0/1/2 select SOUKUP, FLUKA
    and GAUSS_FIT (the energy dict then carries the nuclear tables).
    `carbon_profile` switches on the CarbonPBS lateral profile model of the beams'
    profile_data (bits: 1 sigma override, 2 overall weight). With a biological
    model `bio` (the dict of subsecondpbs_b200._lib.bio_desc) the result also holds
    'bio_acc', its accumulators float64 [4][Z][Y][X]."""
    from subsecondpbs_b200 import _lib as P
    from subsecondpbs_b200.cudaCalDoseRTD import _with_luts

    lib = load()
    beams = beams if beams is not None else [case["beam"]]
    energy = _with_luts(case["energy"], None)
    dd = case["dose_dims"]
    dose_arr = np.zeros((dd[2], dd[1], dd[0]), dtype=np.float64)
    if initial is not None:
        dose_arr += np.asarray(initial, dtype=np.float64).reshape(dose_arr.shape)
    descs, keep = [], []
    for b in beams:
        d, k = P.beam_desc(b)
        descs.append(d)
        keep.append(k)
    arr = (P.PbsBeamDesc * len(descs))(*descs)
    ed, ke = P.energy_desc(energy)
    ct = np.ascontiguousarray(np.asarray(case["ct"], dtype=np.float32))
    cap = None
    bufs = {}
    if capture:
        pl = plan(case, beams[-1])
        S, L = pl["steps"], pl["num_layers"]
        rays = pl["ray_x"] * pl["ray_y"]
        pad = pl["pitch_x"] * pl["pitch_y"]
        tiles = pl["tiles_x"] * pl["tiles_y"]
        bufs = {
            "density": np.zeros((S, pl["ray_y"], pl["ray_x"])), "wepl": np.zeros((S, pl["ray_y"], pl["ray_x"])),
            "first_inside": np.zeros((pl["ray_y"], pl["ray_x"]), np.int32),
            "first_outside": np.zeros((pl["ray_y"], pl["ray_x"]), np.int32),
            "wepl_min": np.zeros(S), "beam_ints": np.zeros(4, np.int32),
            "ray_weights": np.zeros((L, pl["ray_y"], pl["ray_x"])), "entry_sigma": np.zeros((L, 2), np.float32),
            "layer_ints": np.zeros((L, 8), np.int32), "layer_box": np.zeros((L, 6), np.int32),
            "hist": np.zeros((L, 34), np.int32), "batched": np.zeros((L, 33), np.int32),
            "bev": np.zeros((S, pl["bev_y"], pl["bev_x"])),
        }
        if capture_layers:
            bufs["idd"] = np.zeros((L, S, pl["pitch_y"], pl["pitch_x"]))
            bufs["rsigma"] = np.zeros((L, S, pl["pitch_y"], pl["pitch_x"]))
            bufs["codes"] = np.zeros((L, S, pl["tiles_y"], pl["tiles_x"]), np.uint8)
        if nuclear_model >= 0 and pl["nuc_x"] > 0:
            ny, nx = pl["nuc_y"], pl["nuc_x"]
            bufs["nuc_hist"] = np.zeros((L, 34), np.int32)
            bufs["nuc_batched"] = np.zeros((L, 33), np.int32)
            bufs["nuc_bev"] = np.zeros((S, pl["nuc_bev_y"], pl["nuc_bev_x"]))
            bufs["ray_to_nuc"] = np.zeros((pl["ray_y"], pl["ray_x"]), np.int32)
            if capture_layers:
                bufs["nuc_idd"] = np.zeros((L, S, ny, nx))
                bufs["nuc_rsigma"] = np.zeros((L, S, ny, nx))
                bufs["nuc_codes"] = np.zeros((L, S, ny // 8, nx // 32), np.uint8)
        cap = OracleCapture()
        types = {n: t for n, t in OracleCapture._fields_}
        for name, a in bufs.items():
            setattr(cap, name, a.ctypes.data_as(types[name]))
        bufs["plan"] = pl
    lib.oracle_set_carbon_profile(int(carbon_profile))
    bio_acc = None
    if bio:
        bd_bio, keep_bio = P.bio_desc(bio)
        bio_acc = np.zeros((4, dd[2], dd[1], dd[0]), np.float64)
        lib.oracle_set_bio(C.byref(bd_bio), bio_acc.ctypes.data_as(_DP))
    rc = lib.oracle_dose_nuclear(ct.ctypes.data_as(_FP), P.int3(case["ct_dims"]), P.float3(case["ct_resolution"]),
                                 P.float3(case["ct_corner"]), dose_arr.ctypes.data_as(_DP), P.int3(dd),
                                 P.float3(case["dose_resolution"]), P.float3(case["dose_corner"]), arr, len(descs),
                                 C.byref(ed), int(ct_type), int(bool(compat_bev_z_shift)), int(nuclear_model),
                                 int(threads), C.byref(cap) if cap is not None else None)
    lib.oracle_set_carbon_profile(0)
    lib.oracle_set_bio(None, None)
    _err(rc)
    if cap is not None:
        bufs["superpose_fma"] = cap.superpose_fma
        bufs["nuc_superpose_fma"] = cap.nuc_superpose_fma
    del keep, ke
    out = {"dose": dose_arr, "capture": bufs}
    if bio_acc is not None:
        out["bio_acc"] = bio_acc
        del keep_bio
    return out


def bio_map(bio: dict, acc: np.ndarray, name: str) -> np.ndarray:
    """The map `name` ('dose', 'letd', 'rbe', 'rbe_dose', 'alpha', 'beta', 'z1d') of the
    oracle's biological accumulators, float64 [Z][Y][X]."""
    from subsecondpbs_b200 import _lib as P

    lib = load()
    m, keep = P.bio_desc(bio)
    acc = np.ascontiguousarray(acc, np.float64)
    n = acc[0].size
    out = np.zeros(acc.shape[1:], np.float64)
    lib.oracle_bio_map(C.byref(m), acc.ctypes.data_as(_DP), n, P.BIO_MAPS[name], out.ctypes.data_as(_DP))
    del keep
    return out


def radius_bucket(m: float) -> int:
    return int(load().oracle_radius_bucket(C.c_float(m)))


def batch(hist) -> tuple[np.ndarray, np.ndarray]:
    h = np.ascontiguousarray(np.asarray(hist, dtype=np.int32))
    b = np.zeros(33, np.int32)
    m = np.zeros(34, np.int32)
    load().oracle_batch(h.ctypes.data_as(_IP), b.ctypes.data_as(_IP), m.ctypes.data_as(_IP))
    return b, m
