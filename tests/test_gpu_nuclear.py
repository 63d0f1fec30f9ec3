"""Nuclear halo branch (halo lattice IDD/sigma, halo tile superposition and halo
transfer) against the oracle on the same inputs."""
import numpy as np
import pytest

from subsecondpbs_b200 import _lib as L
from subsecondpbs_b200 import phantoms, tables
from _parity import (DOSE_TOL_FRAC_DMAX, GAMMA_PASS_MIN, assert_nuclear_parity, assert_stage_parity,
                     gamma_pass_rate, max_rel_err, nuclear_report, oracle_run, run_gpu, stage_report)

pytestmark = pytest.mark.gpu


def _with_halo_tables(case):
    out = dict(case)
    out["energy"] = tables.synthetic_nuclear_tables(case["energy"])
    return out


def _dose_checks(dose, ref, spacing):
    err = max_rel_err(dose, ref)
    assert err < DOSE_TOL_FRAC_DMAX, err
    assert gamma_pass_rate(dose, ref, spacing) >= GAMMA_PASS_MIN
    assert err < 1e-4, err


def test_gauss_fit_halo_stage_parity(hetero_small_case):
    case = _with_halo_tables(hetero_small_case)
    eng = run_gpu(case, nuclear_model=L.NUCLEAR_GAUSS_FIT)
    r = oracle_run(case, capture=True, capture_layers=True, nuclear_model=L.NUCLEAR_GAUSS_FIT)
    cap = r["capture"]
    assert_stage_parity(stage_report(eng, cap))
    rep = nuclear_report(eng, cap)
    assert rep["fma_oracle"] > 0
    assert_nuclear_parity(rep)
    assert eng.beam_stats()["kernel_launches"] == 6 + 7 + 8 + 2
    _dose_checks(eng.read_dose(), r["dose"], case["dose_resolution"])


@pytest.mark.parametrize("model", [L.NUCLEAR_SOUKUP, L.NUCLEAR_FLUKA])
def test_other_halo_models_dose(hetero_small_case, model):
    case = _with_halo_tables(hetero_small_case)
    eng = run_gpu(case, nuclear_model=model, keep_debug=False)
    r = oracle_run(case, nuclear_model=model)
    _dose_checks(eng.read_dose(), r["dose"], case["dose_resolution"])


def test_halo_changes_the_dose(hetero_small_case):
    case = _with_halo_tables(hetero_small_case)
    with_halo = run_gpu(case, nuclear_model=L.NUCLEAR_GAUSS_FIT, keep_debug=False).read_dose()
    without = run_gpu(case, keep_debug=False).read_dose()
    assert np.abs(with_halo - without).max() > 1e-3 * without.max()


def test_halo_headline_beam(hetero_case):
    case = _with_halo_tables(hetero_case)
    eng = run_gpu(case, nuclear_model=L.NUCLEAR_GAUSS_FIT, keep_debug=False)
    r = oracle_run(case, nuclear_model=L.NUCLEAR_GAUSS_FIT)
    _dose_checks(eng.read_dose(), r["dose"], case["dose_resolution"])


def test_halo_needs_spot_lattice_and_tables(hetero_small_case):
    from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine

    case = _with_halo_tables(hetero_small_case)
    eng = DoseEngine(0)
    eng.set_energy(case["energy"])
    eng.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    eng.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    with pytest.raises(L.PbsError) as e:
        eng.add_beam(phantoms.legacy_beam(case["beam"]), nuclear_correction=True)
    assert e.value.code == L.PBS_ERR_UNSUPPORTED and "raw spot lattice" in str(e.value)
    plain = DoseEngine(0)
    plain.set_energy(hetero_small_case["energy"])
    plain.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    plain.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    with pytest.raises(L.PbsError) as e:
        plain.add_beam(case["beam"], nuclear_correction=True)
    assert e.value.code == L.PBS_ERR_UNSUPPORTED and "nuclear_weight" in str(e.value)
