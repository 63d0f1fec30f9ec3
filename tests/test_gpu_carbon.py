"""Carbon-ion plans with the nuclear halo (the 512x512x200 CT at 1 mm, three
beams of 40 layers 120-400 MeV/u): a reduced plan against the oracle stage by
stage, and the full-size plan through its size-independent properties (beam
additivity, finite non-negative dose) plus one full beam against the oracle."""
import numpy as np
import pytest

from subsecondpbs_b200 import phantoms

from _parity import gamma_pass_rate, max_rel_err, oracle_run, run_gpu

pytestmark = pytest.mark.gpu

HALO = 2  # GAUSS_FIT


def test_reduced_carbon_plan_matches_the_oracle():
    case = phantoms.carbon_case(dims=(128, 128, 64), res=(2.0, 2.0, 2.0), n_layers=8, spots_per_layer=60)
    eng = run_gpu(case, beams=case["beams"], keep_debug=False, nuclear_model=HALO)
    r = oracle_run(case, beams=case["beams"], nuclear_model=HALO)
    dose = eng.read_dose()
    err = max_rel_err(dose, r["dose"])
    assert err < 5e-3, err
    assert gamma_pass_rate(dose, r["dose"], case["dose_resolution"]) >= 0.999


@pytest.fixture(scope="module")
def config3():
    return phantoms.carbon_case()


def test_config3_plan_is_the_sum_of_its_beams(config3):
    case = config3
    assert sum(int(b["layer_spot_counts"].sum()) for b in case["beams"]) >= 14000
    from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine

    eng = DoseEngine(0, nuclear_model=HALO)
    eng.set_energy(case["energy"])
    eng.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    eng.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    singles = []
    for b in case["beams"]:
        eng.reset_dose()
        eng.add_beam(b, nuclear_correction=True)
        singles.append(eng.read_dose64())
    eng.reset_dose()
    for b in case["beams"]:
        eng.add_beam(b, nuclear_correction=True)
    plan = eng.read_dose64()
    eng.close()
    total = np.sum(singles, axis=0)
    assert np.isfinite(plan).all() and plan.min() >= 0.0 and plan.max() > 0.0
    assert np.abs(plan - total).max() <= 2e-5 * total.max()


def test_config3_beam_matches_the_oracle(config3):
    case = config3
    beam = case["beams"][1]
    eng = run_gpu(case, beams=[beam], keep_debug=False, nuclear_model=HALO)
    r = oracle_run(case, beams=[beam], nuclear_model=HALO)
    dose = eng.read_dose()
    err = max_rel_err(dose, r["dose"])
    print(f"config-3 beam: max err {err:.3g} of Dmax")
    assert err < 5e-3, err
    assert gamma_pass_rate(dose, r["dose"], case["dose_resolution"]) >= 0.999
