"""The CUDA library against outputs of the reference itself (tests/golden, see
test_cpu_golden.py), with the reference's BEV depth indexing reproduced
(PBS_OPT_COMPAT_BEV_Z_SHIFT)."""
import numpy as np
import pytest

from _parity import gamma_pass_rate, run_gpu
from test_cpu_golden import PINS, carbon_profile_of, load_case, nuclear_model_of, pinned_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(PINS))
def test_cuda_matches_reference_outputs(name):
    z, meta, case, beam = load_case(name)
    tol, gmin, flips, drop = PINS[name]
    nuc = nuclear_model_of(meta)
    eng = run_gpu(case, beams=[beam], compat=True, keep_debug=False, nuclear_model=nuc,
                  carbon_profile=carbon_profile_of(meta))
    dose = eng.read_dose()
    ref = z["dose"].astype(np.float64)
    assert pinned_err(dose, ref, drop) < tol
    assert gamma_pass_rate(dose, ref, case["dose_resolution"]) >= gmin
    moved = nuc_moved = 0
    for l in range(z["batched"].shape[0]):
        ls = eng.layer_stats(l)
        moved += int(np.abs(np.asarray(ls["batched_counts"]) - z["batched"][l]).sum()) // 2
        if nuc is not None:
            nuc_moved += int(np.abs(np.asarray(ls["nuc_batched_counts"]) - z["nuc_batched"][l]).sum()) // 2
    assert moved <= flips
    assert nuc_moved <= flips
