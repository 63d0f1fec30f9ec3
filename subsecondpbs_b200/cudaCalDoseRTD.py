"""Python face of the dose pipeline with the reference pybind module's names.

Mirrors `cudaCalDoseRTD` (src/bindings/raytracedicom_pybind.cpp:2054-2313):
`raytracedicom_wrapper(ct, ct_dims, ct_resolution, ct_corner, dose_dims,
dose_resolution, dose_corner, beam, energy, gpu_id=0, nuclear_correction=False,
verbose=0, tables_dir="tables/")` returns the dose as float32 [Z][Y][X]. The beam
and energy dicts take the reference's keys; density / stopping-power /
radiation-length LUTs missing from `energy` are read from `tables_dir`, as the
reference does (raytracedicom_pybind.cpp:1846-1847).

Every call runs on the GPU through libsubsecondpbs_b200.so; errors raise
RuntimeError (`_lib.PbsError`) like the reference's pybind translation of
std::runtime_error.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _lib

__all__ = ["raytracedicom_wrapper", "DoseEngine", "cuFinalDose", "calcDose", "cuCalDose", "cuCalDose3",
           "debug_build_carbonpbs_context"]


def _with_luts(energy: dict, tables_dir: str | Path | None) -> dict:
    need = [k for k in ("density_vector", "sp_vector", "rrl_vector") if k not in energy]
    if not need:
        return energy
    from .tables import energy_reader

    if tables_dir is None or not (Path(tables_dir) / "density_Schneider2000_adj.txt").exists():
        from .tables import hu_luts

        extra = hu_luts()
    else:
        extra = energy_reader(tables_dir)
    out = dict(energy)
    for key in ("density", "sp", "rrl"):
        if f"{key}_vector" not in out:
            out[f"{key}_vector"] = extra[f"{key}_vector"]
            out[f"n_{key}_samples"] = extra[f"n_{key}_samples"]
            out[f"{key}_scale_fact"] = extra[f"{key}_scale_fact"]
    return out


def _check_beam(beam: dict) -> None:
    sub = np.asarray(beam["subspot_data"])
    if sub.ndim != 3 or sub.shape[2] != 5:
        raise RuntimeError("subspot_data must have shape (num_layers, max_subspots_per_layer, 5)")
    n_layers = sub.shape[0]
    if len(np.asarray(beam["energies"]).reshape(-1)) != n_layers:
        raise RuntimeError("beam.energies length must equal subspot_data.shape[0] (num_layers)")
    if np.asarray(beam["spot_sigmas"]).reshape(-1, 2).shape[0] != n_layers:
        raise RuntimeError("beam.spot_sigmas length must equal num_layers")
    lc = beam.get("layer_longitudinal_cutoffs")
    if lc is not None and len(np.asarray(lc).reshape(-1)) != n_layers:
        raise RuntimeError("beam.layer_longitudinal_cutoffs length must equal num_layers")


def raytracedicom_wrapper(ct, ct_dims, ct_resolution, ct_corner, dose_dims, dose_resolution, dose_corner,
                          beam: dict, energy: dict, gpu_id: int = 0, nuclear_correction: bool = False,
                          verbose: int = 0, tables_dir: str = "tables/") -> np.ndarray:
    """Dose of one beam as float32 [Z][Y][X] (raytracedicom_pybind.cpp:1679-1871)."""
    lib = _lib.load()
    ct_arr = np.ascontiguousarray(np.asarray(ct, dtype=np.float32))
    if ct_arr.size != int(np.prod(ct_dims)):
        raise RuntimeError("ct buffer size does not match ct_dims")
    _check_beam(beam)
    energy = _with_luts(energy, tables_dir)
    dose = np.zeros((int(dose_dims[2]), int(dose_dims[1]), int(dose_dims[0])), dtype=np.float32)
    bd, keep_b = _lib.beam_desc(beam)
    ed, keep_e = _lib.energy_desc(energy)
    rc = lib.pbs_subsecond_wrapper(
        ct_arr.ctypes.data_as(C.POINTER(C.c_float)), _lib.int3(ct_dims), _lib.float3(ct_resolution),
        _lib.float3(ct_corner), dose.ctypes.data_as(C.POINTER(C.c_float)), _lib.int3(dose_dims),
        _lib.float3(dose_resolution), _lib.float3(dose_corner), C.byref(bd), 1, C.byref(ed), int(gpu_id),
        int(bool(nuclear_correction)), int(verbose))
    del keep_b, keep_e
    _lib.check(rc)
    if not np.all(np.isfinite(dose)):
        raise RuntimeError("raytracedicom_wrapper produced non-finite dose values")
    return dose


class DoseEngine:
    """Resident dose context on one GPU (lookup tables, CT and FP64 dose grid stay
    on the device between calls). Wraps the pbs_context_* C ABI."""

    def __init__(self, gpu_id: int = 0, compat_bev_z_shift: bool = False, stage_timing: bool = False,
                 keep_debug: bool = False, layer_budget_mib: int | None = None, ct_input_type: int | None = None,
                 nuclear_model: int | None = None, carbon_profile: int = 0):
        self._lib = _lib.load()
        h = C.c_void_p()
        _lib.check(self._lib.pbs_context_create(int(gpu_id), C.byref(h)))
        self._h = h
        self.gpu_id = gpu_id
        self.set_option(_lib.PBS_OPT_COMPAT_BEV_Z_SHIFT, int(compat_bev_z_shift))
        self.set_option(_lib.PBS_OPT_STAGE_TIMING, int(stage_timing))
        self.set_option(_lib.PBS_OPT_KEEP_DEBUG, int(keep_debug))
        if layer_budget_mib is not None:
            self.set_option(_lib.PBS_OPT_LAYER_BUDGET_MIB, int(layer_budget_mib))
        if ct_input_type is not None:
            self.set_option(_lib.PBS_OPT_CT_INPUT_TYPE, int(ct_input_type))
        if nuclear_model is not None:
            self.set_option(_lib.PBS_OPT_NUCLEAR_MODEL, int(nuclear_model))
        if carbon_profile:
            self.set_option(_lib.PBS_OPT_CARBON_PROFILE, int(carbon_profile))
        self.dose_dims = None

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.pbs_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, option: int, value: int) -> None:
        _lib.check(self._lib.pbs_context_set_option(self._h, int(option), int(value)))

    def set_energy(self, energy: dict, tables_dir: str | None = None) -> None:
        ed, keep = _lib.energy_desc(_with_luts(energy, tables_dir))
        _lib.check(self._lib.pbs_context_set_energy(self._h, C.byref(ed)))
        del keep

    def set_ct(self, ct, dims, resolution, corner) -> None:
        """`ct` is a float32 [Z][Y][X] numpy array (host) or a CUDA torch tensor."""
        on_dev, ptr, keep = self._ptr(ct, np.float32)
        _lib.check(self._lib.pbs_context_set_ct(self._h, ptr, on_dev, _lib.int3(dims), _lib.float3(resolution),
                                                _lib.float3(corner)))
        del keep

    def set_dose_grid(self, dims, resolution, corner) -> None:
        _lib.check(self._lib.pbs_context_set_dose_grid(self._h, _lib.int3(dims), _lib.float3(resolution),
                                                       _lib.float3(corner)))
        self.dose_dims = tuple(int(d) for d in dims)

    def reset_dose(self, initial=None) -> None:
        if initial is None:
            _lib.check(self._lib.pbs_context_reset_dose(self._h, None, 0))
            return
        on_dev, ptr, keep = self._ptr(initial, np.float32)
        _lib.check(self._lib.pbs_context_reset_dose(self._h, ptr, on_dev))
        del keep

    def add_beam(self, beam, nuclear_correction: bool = False) -> None:
        """Enqueue the dose of `beam` (a beam dict or a `prepare_beam` result)."""
        bd, keep = beam if isinstance(beam, tuple) else _lib.beam_desc(beam)
        _lib.check(self._lib.pbs_context_add_beam(self._h, C.byref(bd), int(bool(nuclear_correction))))
        del keep

    def adjoint_beam(self, beam, grad_dose, n_spots: int | None = None) -> np.ndarray:
        """Gradient of <grad_dose, dose of `beam`> with respect to the beam's spot
        weights at their current values (float32 [n_spots], the beam's spot order).
        `grad_dose` is a float64 [Z][Y][X] numpy array or CUDA tensor."""
        if isinstance(beam, tuple):
            bd, keep = beam
        else:
            bd, keep = _lib.beam_desc(beam)
        if n_spots is None:
            n_spots = int(sum(bd.layer_spot_counts[i] for i in range(bd.n_layer_spot_counts)))
        out = np.zeros(n_spots, dtype=np.float32)
        on_dev, ptr, gkeep = self._ptr(grad_dose, np.float64)
        _lib.check(self._lib.pbs_context_adjoint_beam(self._h, C.byref(bd), ptr, on_dev,
                                                      out.ctypes.data_as(C.POINTER(C.c_float)), n_spots))
        del keep, gkeep
        return out

    def set_bio_model(self, model: dict | None) -> None:
        """Biological model for the maps on top of the dose (see _lib.bio_desc for
        the dict); None clears it. The accumulators restart at zero."""
        m, keep = _lib.bio_desc(model)
        _lib.check(self._lib.pbs_context_set_bio_model(self._h, C.byref(m)))
        del keep

    def read_bio_map(self, name: str, out=None) -> np.ndarray:
        """One biological map ('dose', 'letd', 'rbe', 'rbe_dose', 'alpha', 'beta',
        'z1d') as float32 [Z][Y][X]; a CUDA float32 tensor `out` is filled on the
        device instead."""
        code = _lib.BIO_MAPS[name]
        if out is not None and hasattr(out, "data_ptr"):
            _lib.check(self._lib.pbs_context_read_bio_map(self._h, code, C.c_void_p(out.data_ptr()), 1))
            return out
        dd = self.dose_dims
        res = np.empty((dd[2], dd[1], dd[0]), np.float32)
        _lib.check(self._lib.pbs_context_read_bio_map(self._h, code, res.ctypes.data_as(C.c_void_p), 0))
        return res

    def influence_row_norms(self, beam, voxels=None, spot_begin: int = 0, spot_count: int | None = None,
                            nuclear_correction: bool = False) -> np.ndarray:
        """Row norms of the dose-influence matrix (CarbonPBS cuCalDoseNorm): for each
        voxel the sum over the spots of its squared dose per unit spot weight.
        `voxels` are linear indices (z*Y + y)*X + x (float32 [n] result); without
        them the result is the whole grid, float32 [Z][Y][X]. The context's dose
        accumulator is left at zero."""
        bd, keep = beam if isinstance(beam, tuple) else _lib.beam_desc(beam)
        n_spots = int(sum(bd.layer_spot_counts[i] for i in range(bd.n_layer_spot_counts)))
        if spot_count is None:
            spot_count = n_spots - int(spot_begin)
        if voxels is None:
            dd = self.dose_dims
            out = np.empty((dd[2], dd[1], dd[0]), np.float32)
            vptr, nv = None, 0
        else:
            vox = np.ascontiguousarray(np.asarray(voxels, np.int64).reshape(-1))
            out = np.empty(vox.size, np.float32)
            vptr, nv = vox.ctypes.data_as(C.c_void_p), vox.size
        _lib.check(self._lib.pbs_context_influence_row_norms(
            self._h, C.byref(bd), int(bool(nuclear_correction)), int(spot_begin), int(spot_count), vptr, nv,
            out.ctypes.data_as(C.c_void_p)))
        del keep
        return out

    def influence_csc(self, beam, spot_begin: int = 0, spot_count: int | None = None, threshold: float = 0.0,
                      nuclear_correction: bool = False, capacity: int | None = None):
        """Spot-preserving dose-influence matrix of spots [spot_begin, spot_begin +
        spot_count) as a scipy CSC matrix of shape (voxels, spot_count): column j is
        the dose per unit weight of spot spot_begin + j under the beam's own plan,
        rows are linear voxel indices (z*Y + y)*X + x, entries |dose| > threshold.
        The context's dose accumulator is left at zero. Without `capacity` the
        export runs twice when the first guess of its size is short."""
        import scipy.sparse as sp

        bd, keep = beam if isinstance(beam, tuple) else _lib.beam_desc(beam)
        n_spots = int(sum(bd.layer_spot_counts[i] for i in range(bd.n_layer_spot_counts)))
        if spot_count is None:
            spot_count = n_spots - int(spot_begin)
        n_vox = int(np.prod(self.dose_dims))
        cap = int(capacity) if capacity is not None else max(1 << 16, 4096 * int(spot_count))
        col_ptr = np.zeros(int(spot_count) + 1, dtype=np.int64)
        nnz = C.c_longlong(0)
        while True:
            rows = np.empty(cap, dtype=np.int32)
            vals = np.empty(cap, dtype=np.float32)
            rc = self._lib.pbs_context_influence_csc(
                self._h, C.byref(bd), int(bool(nuclear_correction)), int(spot_begin), int(spot_count),
                float(threshold), col_ptr.ctypes.data_as(C.POINTER(C.c_longlong)), rows.ctypes.data_as(C.c_void_p),
                vals.ctypes.data_as(C.c_void_p), cap, C.byref(nnz))
            if rc == _lib.PBS_ERR_INVALID_ARGUMENT and nnz.value > cap and capacity is None:
                cap = int(nnz.value)
                continue
            _lib.check(rc)
            break
        del keep
        n = int(nnz.value)
        return sp.csc_matrix((vals[:n], rows[:n], col_ptr), shape=(n_vox, int(spot_count)))

    @staticmethod
    def prepare_beam(beam: dict):
        """Convert a beam dict to its C descriptor once (for repeated add_beam calls)."""
        return _lib.beam_desc(beam)

    def read_dose(self, out=None):
        """Dose as float32 [Z][Y][X]: into `out` (numpy or CUDA tensor) or a new array."""
        if out is None:
            out = np.empty((self.dose_dims[2], self.dose_dims[1], self.dose_dims[0]), dtype=np.float32)
        on_dev, ptr, keep = self._ptr(out, np.float32)
        _lib.check(self._lib.pbs_context_read_dose(self._h, ptr, on_dev))
        return out

    def read_dose64(self, out=None):
        """The FP64 accumulator [Z][Y][X] into `out` (numpy or CUDA float64 tensor)."""
        if out is None:
            out = np.empty((self.dose_dims[2], self.dose_dims[1], self.dose_dims[0]), dtype=np.float64)
        on_dev, ptr, keep = self._ptr(out, np.float64)
        _lib.check(self._lib.pbs_context_read_dose64(self._h, ptr, on_dev))
        return out

    def synchronize(self) -> None:
        _lib.check(self._lib.pbs_context_synchronize(self._h))

    @property
    def stream_handle(self) -> int:
        return int(self._lib.pbs_context_stream(self._h) or 0)

    @property
    def dose_device_ptr(self) -> int:
        return int(self._lib.pbs_context_dose_device_ptr(self._h) or 0)

    def beam_stats(self) -> dict:
        s = _lib.PbsBeamStats()
        _lib.check(self._lib.pbs_context_beam_stats(self._h, C.byref(s)))
        return _lib.struct_to_dict(s)

    def layer_stats(self, layer: int) -> dict:
        s = _lib.PbsLayerStats()
        _lib.check(self._lib.pbs_context_layer_stats(self._h, int(layer), C.byref(s)))
        return _lib.struct_to_dict(s)

    def stage_times(self) -> dict:
        buf = (C.c_float * len(_lib.STAGES))()
        _lib.check(self._lib.pbs_context_stage_times(self._h, buf, len(_lib.STAGES)))
        return dict(zip(_lib.STAGES, list(buf)))

    def debug(self, which: int, layer: int = 0, shape=None, dtype=np.float32) -> np.ndarray:
        out = np.empty(shape, dtype=dtype)
        _lib.check(self._lib.pbs_context_debug_copy(self._h, int(which), int(layer),
                                                    out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    @staticmethod
    def _ptr(a, dtype):
        if hasattr(a, "data_ptr") and getattr(a, "is_cuda", False):
            if not a.is_contiguous():
                raise ValueError("device tensors must be contiguous")
            return 1, C.c_void_p(a.data_ptr()), a
        arr = np.ascontiguousarray(np.asarray(a, dtype=dtype))
        if arr is not a and isinstance(a, np.ndarray) and a.dtype == dtype and a.flags.c_contiguous:
            arr = a
        return 0, arr.ctypes.data_as(C.c_void_p), arr


def fp32_peak_tflops(gpu_id: int = 0) -> float:
    """Measured FP32 FMA throughput of the GPU (TFLOP/s)."""
    lib = _lib.load()
    v = C.c_double(0.0)
    _lib.check(lib.pbs_measure_fp32_peak(int(gpu_id), C.byref(v)))
    return float(v.value)


def plan_beam(beam: dict, energy: dict, ct_dims, ct_resolution, ct_corner, dose_dims, dose_resolution,
              dose_corner, tables_dir: str | None = None, with_lattice: bool = False) -> dict:
    """Host-side beam plan (no GPU needed): ray grid, tracer geometry, per-layer
    energy parameters and optionally the dense spot lattice."""
    lib = _lib.load()
    energy = _with_luts(energy, tables_dir)
    bd, keep_b = _lib.beam_desc(beam)
    ed, keep_e = _lib.energy_desc(energy)
    st = _lib.PbsBeamStats()
    n_layers = len(np.asarray(beam["energies"]).reshape(-1))
    lp = np.zeros((n_layers, 8), dtype=np.float32)
    rc = lib.pbs_plan_beam(C.byref(bd), C.byref(ed), _lib.int3(ct_dims), _lib.float3(ct_resolution),
                           _lib.float3(ct_corner), _lib.int3(dose_dims), _lib.float3(dose_resolution),
                           _lib.float3(dose_corner), C.byref(st), lp.ctypes.data_as(C.POINTER(C.c_float)), None, 0)
    _lib.check(rc)
    out = _lib.struct_to_dict(st)
    out["layer_params"] = lp
    if with_lattice and st.conv_mode == 0:
        lat = np.zeros((n_layers, st.lattice_dims[1], st.lattice_dims[0]), dtype=np.float32)
        rc = lib.pbs_plan_beam(C.byref(bd), C.byref(ed), _lib.int3(ct_dims), _lib.float3(ct_resolution),
                               _lib.float3(ct_corner), _lib.int3(dose_dims), _lib.float3(dose_resolution),
                               _lib.float3(dose_corner), C.byref(st), None,
                               lat.ctypes.data_as(C.POINTER(C.c_float)), lat.size)
        _lib.check(rc)
        out["lattice"] = lat
    del keep_b, keep_e
    return out


# CarbonPBS-contract entry points (raytracedicom_pybind.cpp:2088-2313).
from .carbonpbs import calcDose, cuCalDose, cuCalDose3, cuFinalDose, debug_build_carbonpbs_context  # noqa: E402,F401
