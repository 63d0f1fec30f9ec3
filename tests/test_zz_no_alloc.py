"""The allocation-free CPB fluence entry point against the context path on the same
beam. Collected last so that it also runs after everything else the suite did on
the device."""
import ctypes as C

import numpy as np
import pytest

from subsecondpbs_b200 import _lib as L
from subsecondpbs_b200 import phantoms
from _parity import run_gpu

pytestmark = pytest.mark.gpu


def _entry():
    lib = L.load()
    f = lib.pbs_cpb_fluence_no_alloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_float),
                  C.c_void_p, C.c_void_p]
    return f


def test_cpb_fluence_no_alloc_matches_context(hetero_small_case):
    import torch

    beam = phantoms.legacy_beam(hetero_small_case["beam"])
    eng = run_gpu(hetero_small_case, beams=[beam])
    st = eng.beam_stats()
    assert st["conv_mode"] == 1
    nl = st["num_layers"]
    rx, ry = st["ray_dims"]
    ref = eng.debug(L.PBS_DBG_RAY_WEIGHTS, 0, (nl, ry, rx))
    assert ref.max() > 0

    sub = np.ascontiguousarray(beam["subspot_data"], np.float32)
    torch.cuda.set_device(0)
    d_sub = torch.from_numpy(sub).to("cuda:0")
    d_out = torch.full((nl, ry, rx), float("nan"), dtype=torch.float32, device="cuda:0")
    f = _entry()
    dims = (C.c_int * 2)(rx, ry)
    corner = (C.c_float * 2)(*st["cpb_corner"])
    res = (C.c_float * 2)(*st["cpb_resolution"])
    # Two calls in a row: the second must not see the first one's scratch.
    for _ in range(2):
        rc = f(d_sub.data_ptr(), sub.shape[1], nl, dims, corner, res, d_out.data_ptr(), None)
        assert rc == 0, L.load().pbs_last_error()
        torch.cuda.synchronize()
        out = d_out.cpu().numpy()
        assert np.isfinite(out).all()
        assert float(np.abs(out - ref).max() / ref.max()) < 1e-5
        d_out.fill_(float("nan"))


def test_cpb_fluence_no_alloc_rejects_oversized_grid():
    f = _entry()
    dims = (C.c_int * 2)(1024, 1024)
    corner = (C.c_float * 2)(0.0, 0.0)
    res = (C.c_float * 2)(1.0, 1.0)
    # 1024 x 1024 x 2 layers is twice the static scratch: refused before any launch.
    rc = f(C.c_void_p(16), 1, 2, dims, corner, res, C.c_void_p(16), None)
    assert rc == L.PBS_ERR_INVALID_ARGUMENT
    msg = L.load().pbs_last_error()
    msg = msg.decode() if isinstance(msg, bytes) else str(msg)
    assert "static scratch" in msg


def test_cpb_fluence_no_alloc_rejects_launch_limits():
    f = _entry()
    corner = (C.c_float * 2)(0.0, 0.0)
    res = (C.c_float * 2)(1.0, 1.0)
    # 70000 layers of one ray fit the scratch but not the kernels' grid: refused before any launch.
    rc = f(C.c_void_p(16), 1, 70000, (C.c_int * 2)(1, 1), corner, res, C.c_void_p(16), None)
    assert rc == L.PBS_ERR_INVALID_ARGUMENT
    msg = L.load().pbs_last_error()
    msg = msg.decode() if isinstance(msg, bytes) else str(msg)
    assert "launch limits" in msg
