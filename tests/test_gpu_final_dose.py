"""The legacy cudaFinalDose symbol: the reference's stub zeroes the device dose
grid when the beam points at the ROI and leaves it untouched otherwise
(src/algorithms/cuda_final_dose.cu:132-151, 282-298, 370-372)."""
import ctypes as C

import pytest

from subsecondpbs_b200 import _lib as L

pytestmark = pytest.mark.gpu


class V3f(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class V3i(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("z", C.c_int)]


def _call(roi, dose, direction, source):
    lib = L.load()
    f = lib.cudaFinalDose
    f.restype = None
    f.argtypes = [C.c_ulonglong, C.c_void_p, C.c_int, V3f, V3f, V3f, V3f, C.c_float, C.c_float, C.c_int, C.c_int,
                  C.c_void_p, V3i]
    dims = dose.shape
    f(0, roi.data_ptr(), roi.shape[0], V3f(0.2, 0.2, 0.2), V3f(-3.0, -3.0, -3.0), V3f(*direction), V3f(*source),
      100.0, 0.0, 1, 1, dose.data_ptr(), V3i(dims[2], dims[1], dims[0]))


def test_final_dose_zeroes_when_the_beam_points_at_the_roi():
    import torch

    roi = torch.tensor([[10, 10, 10], [20, 20, 20]], dtype=torch.int32, device="cuda:0")
    dose = torch.ones((30, 30, 30), dtype=torch.float32, device="cuda:0")
    _call(roi, dose, (0.0, 0.0, 1.0), (0.0, 0.0, -100.0))
    torch.cuda.synchronize()
    assert float(dose.abs().max()) == 0.0


def test_final_dose_leaves_the_grid_when_the_beam_points_away():
    import torch

    roi = torch.tensor([[10, 10, 10], [20, 20, 20]], dtype=torch.int32, device="cuda:0")
    dose = torch.ones((30, 30, 30), dtype=torch.float32, device="cuda:0")
    _call(roi, dose, (0.0, 0.0, -1.0), (0.0, 0.0, -100.0))
    torch.cuda.synchronize()
    assert float(dose.min()) == 1.0
