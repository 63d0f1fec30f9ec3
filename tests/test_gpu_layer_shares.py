"""Layer sharding of one beam on the GPU: the shares of sharding.assign_layers,
each run as its own beam (the other layers' spots at zero weight), add up to the
whole beam's dose. The reduction across ranks is covered with gloo on the CPU
(test_cpu_sharding.py); here every share runs on the one GPU in turn."""
import numpy as np
import pytest

from subsecondpbs_b200 import sharding
from subsecondpbs_b200.precision import max_rel_err

from _parity import run_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_layer_shares_sum_to_the_beam(hetero_small_case, world):
    eng = run_gpu(hetero_small_case, keep_debug=False)
    whole = eng.read_dose64()
    total = np.zeros_like(whole)
    for layers in sharding.assign_layers(hetero_small_case["beam"], world):
        eng.reset_dose()
        if layers:
            eng.add_beam(sharding.layer_share(hetero_small_case["beam"], layers))
        total += eng.read_dose64()
    # Equal up to the float summation order of the superposition's BEV adds.
    assert max_rel_err(total, whole, thr=0.0) < 1e-5
