"""ctypes binding of libsubsecondpbs_b200.so (include/subsecondpbs.h).

Loading fails loudly when the shared library is missing: there is no CPU
fallback for the dose pipeline.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libsubsecondpbs_b200.so"

PBS_OK = 0
PBS_ERR_INVALID_ARGUMENT = 1
PBS_ERR_GEOMETRY = 2
PBS_ERR_CUDA = 3
PBS_ERR_OUT_OF_MEMORY = 4
PBS_ERR_UNSUPPORTED = 5
PBS_ERR_NOT_READY = 6
PBS_ERR_TIMEOUT = 7

PBS_CT_AUTO, PBS_CT_HU, PBS_CT_HU_PLUS_1000, PBS_CT_DENSITY, PBS_CT_SPR = range(5)

PBS_OPT_COMPAT_BEV_Z_SHIFT = 1
PBS_OPT_STAGE_TIMING = 2
PBS_OPT_LAYER_BUDGET_MIB = 3
PBS_OPT_CT_INPUT_TYPE = 4
PBS_OPT_KEEP_DEBUG = 5
PBS_OPT_NUCLEAR_MODEL = 6
PBS_OPT_CARBON_PROFILE = 7
PBS_BIO_OFF, PBS_BIO_LQ, PBS_BIO_MKM = 0, 1, 2
BIO_MAPS = {"dose": 0, "letd": 1, "rbe": 2, "rbe_dose": 3, "alpha": 4, "beta": 5, "z1d": 6}
NUCLEAR_SOUKUP, NUCLEAR_FLUKA, NUCLEAR_GAUSS_FIT = 0, 1, 2

STAGES = ("trace", "plan", "conv", "idd", "bin", "superpose", "transfer")

PBS_DBG_DENSITY = 1
PBS_DBG_WEPL = 2
PBS_DBG_FIRST_INSIDE = 3
PBS_DBG_FIRST_OUTSIDE = 4
PBS_DBG_WEPL_MIN = 5
PBS_DBG_RAY_WEIGHTS = 6
PBS_DBG_IDD = 7
PBS_DBG_RSIGMA = 8
PBS_DBG_TILE_BINS = 9
PBS_DBG_BEV_DOSE = 10
PBS_DBG_DOSE64 = 11
PBS_DBG_FIRST_PASSIVE = 12
PBS_DBG_NUC_IDD = 13
PBS_DBG_NUC_RSIGMA = 14
PBS_DBG_NUC_TILE_BINS = 15
PBS_DBG_NUC_BEV_DOSE = 16
PBS_DBG_RAY_TO_NUC = 17

_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)


def _arr(t, n):
    return t * n


class PbsBeamDesc(C.Structure):
    _fields_ = [
        ("energies", _FP), ("n_energies", C.c_size_t),
        ("spot_sigmas", _FP), ("n_spot_sigmas", C.c_size_t),
        ("ray_spacing", _arr(C.c_float, 2)),
        ("steps", C.c_uint),
        ("source_dist", _arr(C.c_float, 2)),
        ("spot_offset", _arr(C.c_float, 3)),
        ("spot_delta", _arr(C.c_float, 3)),
        ("max_subspots_per_layer", C.c_int),
        ("subspot_data", _FP), ("n_subspot_data", C.c_size_t),
        ("layer_spot_counts", _IP), ("n_layer_spot_counts", C.c_size_t),
        ("spot_positions", _FP), ("n_spot_positions", C.c_size_t),
        ("spot_positions_are_indices", C.c_int),
        ("spot_weights", _FP), ("n_spot_weights", C.c_size_t),
        ("spot_beam_directions", _FP), ("n_spot_beam_directions", C.c_size_t),
        ("layer_longitudinal_cutoffs", _FP), ("n_layer_longitudinal_cutoffs", C.c_size_t),
        ("water_equivalence", _FP), ("n_water_equivalence", C.c_size_t),
        ("ray_weq_header", _FP), ("n_ray_weq_header", C.c_size_t),
        ("profile_data", _FP), ("n_profile_data", C.c_size_t),
        ("profile_setting", _FP), ("n_profile_setting", C.c_size_t),
        ("beam_para_data", _FP), ("n_beam_para_data", C.c_size_t),
        ("beam_direction", _arr(C.c_float, 3)),
        ("bm_x_direction", _arr(C.c_float, 3)),
        ("bm_y_direction", _arr(C.c_float, 3)),
        ("source_position", _arr(C.c_float, 3)),
        ("sad", C.c_float),
        ("ref_plane_z", C.c_float),
        ("roi_linear_indices", _IP), ("n_roi_linear_indices", C.c_size_t),
        ("profile_energies", _FP), ("n_profile_energies", C.c_size_t),
        ("beam_para_pos", C.c_float),
    ]


class PbsBioModel(C.Structure):
    _fields_ = [
        ("model", C.c_int),
        ("let_table", _FP), ("let_rows", C.c_int), ("let_depths", C.c_int),
        ("let_energies", _FP),
        ("let_depth0", C.c_float), ("let_depth_step", C.c_float),
        ("let_samples", C.c_int),
        ("est_dimension", C.c_float), ("range_shifter", C.c_float),
        ("lq_alpha", _FP), ("lq_beta", _FP), ("z1d", _FP),
        ("n_lq", C.c_int),
        ("lq_log0", C.c_float), ("lq_log_step", C.c_float),
        ("alpha0", C.c_float), ("beta0", C.c_float),
    ]


class PbsEnergyDesc(C.Structure):
    _fields_ = [
        ("n_energy_samples", C.c_int),
        ("n_energies", C.c_int),
        ("energies_per_u", _FP), ("n_energies_per_u", C.c_size_t),
        ("peak_depths", _FP), ("n_peak_depths", C.c_size_t),
        ("scale_facts", _FP), ("n_scale_facts", C.c_size_t),
        ("cidd_matrix", _FP), ("n_cidd_matrix", C.c_size_t),
        ("n_density_samples", C.c_int),
        ("density_scale_fact", C.c_float),
        ("density_vector", _FP), ("n_density_vector", C.c_size_t),
        ("n_sp_samples", C.c_int),
        ("sp_scale_fact", C.c_float),
        ("sp_vector", _FP), ("n_sp_vector", C.c_size_t),
        ("n_rrl_samples", C.c_int),
        ("rrl_scale_fact", C.c_float),
        ("rrl_vector", _FP), ("n_rrl_vector", C.c_size_t),
        ("nuc_weight_matrix", _FP), ("n_nuc_weight_matrix", C.c_size_t),
        ("nuc_sq_sigma_matrix", _FP), ("n_nuc_sq_sigma_matrix", C.c_size_t),
        ("nuclear_tables_aligned_to_primary_axis", C.c_int),
    ]


class PbsBeamStats(C.Structure):
    _fields_ = [
        ("num_layers", C.c_int), ("conv_mode", C.c_int),
        ("ray_dims", _arr(C.c_int, 2)), ("superp_dims", _arr(C.c_int, 2)),
        ("tracer_steps", C.c_int),
        ("lattice_dims", _arr(C.c_int, 2)), ("lattice_delta", _arr(C.c_float, 2)),
        ("lattice_offset", _arr(C.c_float, 2)),
        ("cpb_corner", _arr(C.c_float, 2)), ("cpb_resolution", _arr(C.c_float, 2)),
        ("fan_corner", _arr(C.c_float, 3)), ("fan_delta", _arr(C.c_float, 3)),
        ("source_dist", _arr(C.c_float, 2)),
        ("len_to_mm", C.c_float), ("energy_depth_to_mm", C.c_float), ("max_peak_depth_mm", C.c_float),
        ("first_inside", C.c_int), ("first_outside", C.c_int), ("guaranteed_passive", C.c_int),
        ("transfer_start", _arr(C.c_int, 3)), ("transfer_max", _arr(C.c_int, 3)),
        ("live_tiles", C.c_longlong), ("superpose_fma", C.c_longlong),
        ("kernel_launches", C.c_int), ("layer_chunks", C.c_int),
        ("nuc_dims", _arr(C.c_int, 2)), ("nuc_live_tiles", C.c_longlong), ("nuc_superpose_fma", C.c_longlong),
    ]


class PbsLayerStats(C.Structure):
    _fields_ = [
        ("energy_idx", C.c_float), ("energy_scale_fact", C.c_float), ("peak_depth", C.c_float),
        ("entry_sigma", _arr(C.c_float, 2)),
        ("after_last_step", C.c_int), ("max_first_passive", C.c_int), ("calc_passive", C.c_int),
        ("tile_rad_counts", _arr(C.c_int, 34)), ("batched_counts", _arr(C.c_int, 33)),
        ("live_tiles", C.c_int),
        ("nuc_tile_rad_counts", _arr(C.c_int, 34)), ("nuc_batched_counts", _arr(C.c_int, 33)),
        ("spot_dist", C.c_float),
    ]


def struct_to_dict(s: C.Structure) -> dict:
    out = {}
    for name, _ in s._fields_:
        v = getattr(s, name)
        if isinstance(v, C.Array):
            v = list(v)
        out[name] = v
    return out


class PbsOperatorLayerSpan(C.Structure):
    _fields_ = [("layer_index", C.c_int), ("spot_begin", C.c_int), ("spot_count", C.c_int),
                ("energy", C.c_float), ("longitudinal_cutoff", C.c_float)]


class PbsOperatorBatch(C.Structure):
    _fields_ = [("batch_index", C.c_int), ("spot_begin", C.c_int), ("spot_count", C.c_int),
                ("first_layer_index", C.c_int), ("last_layer_index", C.c_int)]


class PbsServerStats(C.Structure):
    _fields_ = [(n, C.c_longlong) for n in ("submitted", "completed", "failed", "queued", "running", "patient_loads",
                                            "evictions", "slot_releases", "resident_bytes", "slot_bytes",
                                            "peak_bytes", "budget_bytes", "trace_hits", "trace_loads",
                                            "trace_evictions")]


class PbsError(RuntimeError):
    """Raised for a non-zero status of the native library."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[pbs status {code}] {message}")
        self.code = code


_lib = None


def load() -> C.CDLL:
    """Load the native library (building it first if it is missing and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        if os.environ.get("SUBSECONDPBS_NO_BUILD"):
            raise ImportError(f"{LIB_PATH} is missing and building is disabled")
        from . import build as _build

        _build.build()
    lib = C.CDLL(str(LIB_PATH))
    i, p, vp = C.c_int, C.c_void_p, C.c_void_p
    fp, ip3, fp3 = _FP, C.POINTER(C.c_int), _FP
    sig = {
        "pbs_version": (C.c_char_p, []),
        "pbs_last_error": (C.c_char_p, []),
        "pbs_device_count": (i, [C.POINTER(C.c_int)]),
        "pbs_subsecond_wrapper": (i, [fp, ip3, fp3, fp3, fp, ip3, fp3, fp3, C.POINTER(PbsBeamDesc), C.c_size_t,
                                      C.POINTER(PbsEnergyDesc), i, i, i]),
        "pbs_wrapper_copy_bytes": (i, [C.POINTER(C.c_ulonglong)]),
        "pbs_plan_beam": (i, [C.POINTER(PbsBeamDesc), C.POINTER(PbsEnergyDesc), ip3, fp3, fp3, ip3, fp3, fp3,
                              C.POINTER(PbsBeamStats), fp, fp, C.c_size_t]),
        "pbs_context_create": (i, [i, C.POINTER(vp)]),
        "pbs_context_destroy": (i, [vp]),
        "pbs_context_set_option": (i, [vp, i, C.c_longlong]),
        "pbs_context_set_energy": (i, [vp, C.POINTER(PbsEnergyDesc)]),
        "pbs_context_set_ct": (i, [vp, vp, i, ip3, fp3, fp3]),
        "pbs_context_set_dose_grid": (i, [vp, ip3, fp3, fp3]),
        "pbs_context_reset_dose": (i, [vp, vp, i]),
        "pbs_context_add_beam": (i, [vp, C.POINTER(PbsBeamDesc), i]),
        "pbs_context_adjoint_beam": (i, [vp, C.POINTER(PbsBeamDesc), vp, i, fp, C.c_size_t]),
        "pbs_operator_batch_plan": (i, [C.POINTER(PbsBeamDesc), i, vp, i, vp, i, C.POINTER(C.c_int)]),
        "pbs_context_influence_csc": (i, [vp, C.POINTER(PbsBeamDesc), i, C.c_longlong, C.c_longlong, C.c_double,
                                          C.POINTER(C.c_longlong), vp, vp, C.c_longlong, C.POINTER(C.c_longlong)]),
        "pbs_context_influence_row_norms": (i, [vp, C.POINTER(PbsBeamDesc), i, C.c_longlong, C.c_longlong, vp,
                                                C.c_longlong, vp]),
        "pbs_context_set_bio_model": (i, [vp, C.POINTER(PbsBioModel)]),
        "pbs_context_read_bio_map": (i, [vp, i, vp, i]),
        "pbs_context_read_dose": (i, [vp, vp, i]),
        "pbs_context_read_dose64": (i, [vp, vp, i]),
        "pbs_measure_fp32_peak": (i, [i, C.POINTER(C.c_double)]),
        "pbs_context_synchronize": (i, [vp]),
        "pbs_context_stream": (vp, [vp]),
        "pbs_context_dose_device_ptr": (vp, [vp]),
        "pbs_context_beam_stats": (i, [vp, C.POINTER(PbsBeamStats)]),
        "pbs_context_layer_stats": (i, [vp, i, C.POINTER(PbsLayerStats)]),
        "pbs_context_stage_times": (i, [vp, C.POINTER(C.c_float), i]),
        "pbs_context_debug_copy": (i, [vp, i, i, vp, C.c_size_t]),
        "pbs_server_create": (i, [i, i, C.c_longlong, C.POINTER(vp)]),
        "pbs_server_destroy": (i, [vp]),
        "pbs_server_set_option": (i, [vp, i, C.c_longlong]),
        "pbs_server_set_bypass_limit": (i, [vp, C.c_double]),
        "pbs_server_set_trace_cache": (i, [vp, i]),
        "pbs_server_add_energy": (i, [vp, i, C.POINTER(PbsEnergyDesc)]),
        "pbs_server_add_patient": (i, [vp, i, fp, ip3, fp3, fp3, ip3, fp3, fp3]),
        "pbs_server_remove_patient": (i, [vp, i]),
        "pbs_server_submit": (i, [vp, i, i, C.POINTER(PbsBeamDesc), C.c_size_t, i, C.POINTER(C.c_ulonglong)]),
        "pbs_server_wait": (i, [vp, C.c_ulonglong, C.c_double, C.POINTER(C.POINTER(C.c_float)),
                                C.POINTER(C.c_double), C.POINTER(C.c_int)]),
        "pbs_server_release": (i, [vp, C.c_ulonglong]),
        "pbs_server_request_info": (i, [vp, C.c_ulonglong, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                        C.POINTER(C.c_longlong)]),
        "pbs_server_drain": (i, [vp, C.c_double]),
        "pbs_server_stats": (i, [vp, C.POINTER(PbsServerStats)]),
        "pbs_server_now": (C.c_double, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != PBS_OK:
        msg = load().pbs_last_error()
        raise PbsError(rc, msg.decode() if msg else "")


# ---- descriptor construction -------------------------------------------------

def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1))


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1))


def _vec(keep: list, a, kind=np.float32):
    if a is None:
        return None, 0
    arr = _f32(a) if kind == np.float32 else _i32(a)
    keep.append(arr)
    ptr = arr.ctypes.data_as(_FP if kind == np.float32 else _IP)
    return ptr, arr.size


def _set3(dst, v, default=(0.0, 0.0, 0.0)):
    vals = default if v is None else [float(x) for x in np.asarray(v, dtype=np.float64).reshape(-1)[:3]]
    for k in range(3):
        dst[k] = vals[k]


def beam_desc(beam: dict) -> tuple[PbsBeamDesc, list]:
    """PbsBeamDesc from a beam dict with the keys of the reference's pybind module
    (src/bindings/raytracedicom_pybind.cpp:1711-1821). Returns (desc, keepalive)."""
    keep: list = []
    d = PbsBeamDesc()

    def put(name, key, kind=np.float32, value=None):
        a = beam.get(key) if value is None else value
        ptr, n = _vec(keep, a, kind)
        if ptr is not None:
            setattr(d, name, ptr)
            setattr(d, "n_" + name, n)

    put("energies", "energies")
    put("spot_sigmas", "spot_sigmas")
    rs = beam.get("ray_spacing", (0.0, 0.0))
    d.ray_spacing[0], d.ray_spacing[1] = float(rs[0]), float(rs[1])
    d.steps = int(beam.get("steps", 0))
    sd = beam.get("source_dist", (0.0, 0.0))
    d.source_dist[0], d.source_dist[1] = float(sd[0]), float(sd[1])
    _set3(d.spot_offset, beam.get("spot_offset"))
    _set3(d.spot_delta, beam.get("spot_delta"))
    sub = beam.get("subspot_data")
    if sub is not None:
        sub = np.asarray(sub, dtype=np.float32)
        if sub.ndim != 3 or sub.shape[2] != 5:
            raise ValueError("subspot_data must have shape (num_layers, max_subspots_per_layer, 5)")
        d.max_subspots_per_layer = int(sub.shape[1])
        put("subspot_data", None, value=sub)
    put("layer_spot_counts", "layer_spot_counts", np.int32)
    put("spot_positions", "spot_positions")
    d.spot_positions_are_indices = int(bool(beam.get("spot_positions_are_indices", False)))
    put("spot_weights", "spot_weights")
    put("spot_beam_directions", "spot_beam_directions")
    put("layer_longitudinal_cutoffs", "layer_longitudinal_cutoffs")
    put("water_equivalence", "water_equivalence")
    put("ray_weq_header", "ray_weq_header")
    put("profile_data", "profile_data")
    put("profile_setting", "profile_setting")
    put("beam_para_data", "beam_para_data")
    _set3(d.beam_direction, beam.get("beam_direction"), (0.0, 0.0, 1.0))
    _set3(d.bm_x_direction, beam.get("beam_xdir"), (1.0, 0.0, 0.0))
    _set3(d.bm_y_direction, beam.get("beam_ydir"), (0.0, 1.0, 0.0))
    _set3(d.source_position, beam.get("source_position"))
    d.sad = float(beam.get("sad", 0.0))
    d.ref_plane_z = float(beam.get("ref_plane_z", 0.0))
    put("roi_linear_indices", "roi_linear_indices", np.int32)
    put("profile_energies", "profile_energies")
    d.beam_para_pos = float(beam.get("beam_para_pos", 0.0))
    return d, keep


def bio_desc(model: dict | None) -> tuple[PbsBioModel, list]:
    """PbsBioModel from a dict: model ("lq" | "mkm" | None), let_table [rows][depths],
    let_energies, let_depth0, let_depth_step, let_samples, est_dimension,
    range_shifter, lq_alpha / lq_beta (LQ) or z1d (MKM) on the log10(LET) axis
    lq_log0 + i * lq_log_step, alpha0, beta0."""
    keep: list = []
    m = PbsBioModel()
    if not model or model.get("model") in (None, "off"):
        m.model = PBS_BIO_OFF
        return m, keep
    m.model = {"lq": PBS_BIO_LQ, "mkm": PBS_BIO_MKM}[model["model"]]
    let = np.ascontiguousarray(np.asarray(model["let_table"], np.float32))
    if let.ndim != 2:
        raise ValueError("let_table must be [rows][depths]")
    keep.append(let)
    m.let_table = let.ctypes.data_as(_FP)
    m.let_rows, m.let_depths = int(let.shape[0]), int(let.shape[1])

    def arr(key):
        a = np.ascontiguousarray(np.asarray(model[key], np.float32).reshape(-1))
        keep.append(a)
        return a

    e = arr("let_energies")
    if e.size != m.let_rows:
        raise ValueError("let_energies must have one entry per let_table row")
    m.let_energies = e.ctypes.data_as(_FP)
    m.let_depth0 = float(model.get("let_depth0", 0.0))
    m.let_depth_step = float(model["let_depth_step"])
    m.let_samples = int(model.get("let_samples", 5))
    m.est_dimension = float(model.get("est_dimension", 0.0))
    m.range_shifter = float(model.get("range_shifter", 0.0))
    if m.model == PBS_BIO_LQ:
        a, b = arr("lq_alpha"), arr("lq_beta")
        if a.size != b.size:
            raise ValueError("lq_alpha and lq_beta must have the same length")
        m.lq_alpha, m.lq_beta, m.n_lq = a.ctypes.data_as(_FP), b.ctypes.data_as(_FP), int(a.size)
    else:
        z = arr("z1d")
        m.z1d, m.n_lq = z.ctypes.data_as(_FP), int(z.size)
    m.lq_log0 = float(model.get("lq_log0", 0.0))
    m.lq_log_step = float(model.get("lq_log_step", 0.01))
    m.alpha0 = float(model.get("alpha0", 0.0))
    m.beta0 = float(model.get("beta0", 0.0))
    return m, keep


def energy_desc(energy: dict) -> tuple[PbsEnergyDesc, list]:
    """PbsEnergyDesc from an energy dict with the reference pybind keys
    (raytracedicom_pybind.cpp:1824-1847). Returns (desc, keepalive)."""
    keep: list = []
    e = PbsEnergyDesc()
    e.n_energies = int(energy["n_energies"])
    e.n_energy_samples = int(energy["n_energy_samples"])

    def put(name, key):
        a = energy.get(key)
        ptr, n = _vec(keep, a)
        if ptr is not None:
            setattr(e, name, ptr)
            setattr(e, "n_" + name, n)

    put("energies_per_u", "energies_per_u")
    put("peak_depths", "peak_depths")
    put("scale_facts", "scale_facts")
    put("cidd_matrix", "cidd_matrix")
    put("density_vector", "density_vector")
    put("sp_vector", "sp_vector")
    put("rrl_vector", "rrl_vector")
    put("nuc_weight_matrix", "nuc_weight_matrix")
    put("nuc_sq_sigma_matrix", "nuc_sq_sigma_matrix")
    e.n_density_samples = int(energy.get("n_density_samples", e.n_density_vector))
    e.density_scale_fact = float(energy.get("density_scale_fact", 1.0))
    e.n_sp_samples = int(energy.get("n_sp_samples", e.n_sp_vector))
    e.sp_scale_fact = float(energy.get("sp_scale_fact", 1.0))
    e.n_rrl_samples = int(energy.get("n_rrl_samples", e.n_rrl_vector))
    e.rrl_scale_fact = float(energy.get("rrl_scale_fact", 1.0))
    e.nuclear_tables_aligned_to_primary_axis = int(bool(energy.get("nuclear_tables_aligned_to_primary_axis", False)))
    return e, keep


def int3(v) -> C.Array:
    return (C.c_int * 3)(*[int(x) for x in v])


def float3(v) -> C.Array:
    return (C.c_float * 3)(*[float(x) for x in v])
