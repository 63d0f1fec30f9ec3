"""pbs_subsecond_wrapper copies only the CT voxels its beams trace and the dose
voxels they write. Its result must equal the resident-context path, and the
caller's dose must keep its values where the beams add nothing."""
import ctypes as C

import numpy as np
import pytest

from subsecondpbs_b200 import _lib as L
from subsecondpbs_b200 import phantoms, tables
from subsecondpbs_b200.cudaCalDoseRTD import _with_luts
from _parity import run_gpu

pytestmark = pytest.mark.gpu


def _wrapper(case, beams, initial, nuclear=False):
    lib = L.load()
    descs, keep = [], []
    for b in beams:
        d, k = L.beam_desc(b)
        descs.append(d)
        keep.append(k)
    arr = (L.PbsBeamDesc * len(descs))(*descs)
    ed, ke = L.energy_desc(_with_luts(case["energy"], None))
    ct = np.ascontiguousarray(case["ct"], dtype=np.float32)
    dose = np.ascontiguousarray(initial, dtype=np.float32).copy()
    fp = C.POINTER(C.c_float)
    L.check(lib.pbs_subsecond_wrapper(ct.ctypes.data_as(fp), L.int3(case["ct_dims"]), L.float3(case["ct_resolution"]),
                                      L.float3(case["ct_corner"]), dose.ctypes.data_as(fp), L.int3(case["dose_dims"]),
                                      L.float3(case["dose_resolution"]), L.float3(case["dose_corner"]), arr,
                                      len(descs), C.byref(ed), 0, int(nuclear), 0))
    del keep, ke
    return dose


def _same(got, want, initial):
    # Float atomics make repeated runs differ in the last bits inside the dose.
    m = float(np.abs(want - initial).max())
    assert m > 0
    assert float(np.abs(got - want).max()) <= 1e-6 * m, float(np.abs(got - want).max()) / m
    # Where the beams add nothing the caller's values come back exactly, and the
    # beams reach only part of the grid.
    idle = want == initial
    assert np.array_equal(got[idle], initial[idle])
    assert idle.mean() > 0.05


@pytest.mark.parametrize("angles", [(90.0,), (30.0, 200.0)])
def test_wrapper_regions_equal_the_context_path(hetero_small_case, angles):
    case = hetero_small_case
    beams = [phantoms.rotate_beam(case["beam"], a) for a in angles]
    rng = np.random.default_rng(7)
    initial = rng.uniform(0.0, 1e-9, size=case["ct"].shape).astype(np.float32)
    got = _wrapper(case, beams, initial)
    want = run_gpu(case, beams=beams, keep_debug=False, initial=initial).read_dose()
    _same(got, want, initial)


def test_wrapper_regions_with_the_halo(hetero_small_case):
    case = dict(hetero_small_case)
    case["energy"] = tables.synthetic_nuclear_tables(hetero_small_case["energy"])
    initial = np.zeros(case["ct"].shape, np.float32)
    got = _wrapper(case, [case["beam"]], initial, nuclear=True)
    want = run_gpu(case, keep_debug=False, nuclear_model=L.NUCLEAR_GAUSS_FIT).read_dose()
    _same(got, want, initial)


def _wrapper_ct(case, beam, ct):
    """The wrapper on one beam with `ct` given as a numpy array (pageable) or a
    page-locked torch tensor; returns the dose."""
    lib = L.load()
    d, keep = L.beam_desc(beam)
    ed, ke = L.energy_desc(_with_luts(case["energy"], None))
    dose = np.zeros(tuple(reversed(case["dose_dims"])), dtype=np.float32)
    fp = C.POINTER(C.c_float)
    ptr = C.cast(C.c_void_p(ct.data_ptr()), fp) if hasattr(ct, "data_ptr") else ct.ctypes.data_as(fp)
    L.check(lib.pbs_subsecond_wrapper(ptr, L.int3(case["ct_dims"]), L.float3(case["ct_resolution"]),
                                      L.float3(case["ct_corner"]), dose.ctypes.data_as(fp), L.int3(case["dose_dims"]),
                                      L.float3(case["dose_resolution"]), L.float3(case["dose_corner"]), C.byref(d), 1,
                                      C.byref(ed), 0, 0, 0))
    del keep, ke
    return dose


@pytest.mark.parametrize("form", ["hu+1000", "hu", "density"])
def test_page_locked_ct_detects_the_same_type(hetero_small_case, form):
    """A page-locked host CT has its type detected on the device from the same
    samples: the dose equals the one from a pageable copy of the same CT, for
    each of the three types detection can choose."""
    import torch

    case = hetero_small_case
    ct = np.ascontiguousarray(case["ct"], dtype=np.float32)
    if form == "hu":
        ct = ct - 1000.0
    elif form == "density":
        ct = np.clip(ct / 1000.0, 0.0, 2.0).astype(np.float32)
    want = _wrapper_ct(case, case["beam"], ct)
    got = _wrapper_ct(case, case["beam"], torch.from_numpy(ct.copy()).pin_memory())
    m = float(np.abs(want).max())
    assert m > 0
    assert float(np.abs(got - want).max()) <= 1e-6 * m
