"""CarbonPBS lateral profile model (overrideRSigmaFromCarbonProfileKernel and
applyCarbonProfileOverallWeightKernel, src/core/raytracedicom_wrapper.cu:2080-2187;
compiled but switched off in the reference, raytracedicom_wrapper.cu:2813-2814)
against the CPU oracle on identical seeded inputs: the effective sigma override,
the overall IDD weight and both, with the profile rows per layer and on their own
energy axis. Integer work (tile radius histograms, batch counts, superposition
work) must be bit-exact, dose within the path's tolerance."""
import numpy as np
import pytest

from subsecondpbs_b200 import phantoms

from _parity import DOSE_TOL_FRAC_DMAX, assert_stage_parity, max_rel_err, oracle_run, run_gpu, stage_report

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rows", ["layers", "energies"])
@pytest.mark.parametrize("mode", [1, 2, 3])
def test_profile_model_stage_parity(hetero_small_case, mode, rows):
    beam = phantoms.with_carbon_profile(hetero_small_case["beam"], rows=rows)
    eng = run_gpu(hetero_small_case, beams=[beam], carbon_profile=mode)
    r = oracle_run(hetero_small_case, beams=[beam], capture=True, capture_layers=True, carbon_profile=mode)
    assert_stage_parity(stage_report(eng, r["capture"]))
    dose, ref = eng.read_dose(), r["dose"]
    assert max_rel_err(dose, ref) < 1e-4
    # The model changes the dose: it is not the plain pipeline's.
    plain = oracle_run(hetero_small_case, beams=[beam])["dose"]
    assert max_rel_err(plain, ref) > 10 * DOSE_TOL_FRAC_DMAX


def test_profile_switch_off_is_the_plain_pipeline(hetero_small_case):
    beam = phantoms.with_carbon_profile(hetero_small_case["beam"])
    a = run_gpu(hetero_small_case, beams=[beam], keep_debug=False).read_dose()
    b = run_gpu(hetero_small_case, keep_debug=False).read_dose()
    # Equal up to the float summation order of the superposition's BEV adds.
    assert max_rel_err(a, b, thr=0.0) < 1e-6
