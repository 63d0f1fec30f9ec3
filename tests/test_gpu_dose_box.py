"""The dose grid's dirty box: a context that zeroes and converts only the voxels
its beams' transfers can write gives the same doses as a fresh context, through
zeroing resets, initialised resets, host and device readouts, and after the
FP64 grid's device pointer has been handed out."""
import numpy as np
import pytest
import torch

from subsecondpbs_b200 import phantoms
from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine

pytestmark = pytest.mark.gpu

# Two runs of the same beams differ only in the order of float atomics.
SAME_TOL = 2e-5


def _engine(case):
    eng = DoseEngine(0)
    eng.set_energy(case["energy"])
    eng.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    eng.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    return eng


def _alone(case, beams, initial=None):
    eng = _engine(case)
    if initial is not None:
        eng.reset_dose(initial)
    for b in beams:
        eng.add_beam(b)
    d, d64 = eng.read_dose(), eng.read_dose64()
    eng.close()
    return d, d64


def _close(a, b):
    scale = max(float(np.abs(b).max()), 1e-30)
    return float(np.abs(np.asarray(a, np.float64) - b).max()) / scale


def test_zeroing_reset_clears_earlier_beams(hetero_small_case):
    case = hetero_small_case
    a = case["beam"]
    b = phantoms.rotate_beam(a, 90.0)
    ref_b, ref_b64 = _alone(case, [b])
    ref_ab, _ = _alone(case, [a, b])
    eng = _engine(case)
    eng.add_beam(a)
    eng.add_beam(b)
    assert _close(eng.read_dose(), ref_ab) <= SAME_TOL
    eng.reset_dose()
    eng.add_beam(b)
    d = eng.read_dose()
    d64 = eng.read_dose64()
    assert _close(d, ref_b) <= SAME_TOL
    assert _close(d64, ref_b64) <= SAME_TOL
    # Nothing of beam a is left where beam b deposits nothing.
    assert not np.any(d64[ref_b64 == 0.0])
    # The device readout zeroes the whole output buffer, outside the box too.
    out = torch.full(d.shape, float("nan"), dtype=torch.float32, device="cuda:0")
    eng.read_dose(out)
    eng.synchronize()
    assert np.array_equal(out.cpu().numpy(), d)
    eng.close()


def test_initialised_reset_then_zeroing_reset(hetero_small_case):
    case = hetero_small_case
    b = phantoms.rotate_beam(case["beam"], 240.0)
    shape = tuple(reversed(case["dose_dims"]))
    init = np.random.Generator(np.random.PCG64(5)).random(shape, dtype=np.float32)
    ref_b, _ = _alone(case, [b])
    ref_ib, _ = _alone(case, [b], initial=init)
    eng = _engine(case)
    eng.reset_dose(init)
    eng.add_beam(b)
    assert _close(eng.read_dose(), ref_ib) <= SAME_TOL
    # The initial dose covered the whole grid: the next zeroing reset clears all of it.
    eng.reset_dose()
    eng.add_beam(b)
    assert _close(eng.read_dose(), ref_b) <= SAME_TOL
    assert not np.any(eng.read_dose64()[ref_b == 0.0])
    eng.close()


def test_handed_out_pointer_uses_the_whole_grid(hetero_small_case):
    case = hetero_small_case
    a = case["beam"]
    b = phantoms.rotate_beam(a, 120.0)
    ref_b, _ = _alone(case, [b])
    eng = _engine(case)
    eng.add_beam(a)
    assert eng.dose_device_ptr != 0
    eng.reset_dose()
    eng.add_beam(b)
    assert _close(eng.read_dose(), ref_b) <= SAME_TOL
    assert not np.any(eng.read_dose64()[ref_b == 0.0])
    eng.close()
