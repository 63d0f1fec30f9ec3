"""Water-equivalence import transport (the CarbonPBS rayweq contract) on the GPU
against the oracle: the imported depths and densities, the entry and exit steps
and the per-step minimum depth are exact; the rest of the pipeline is held to the
same bar as a CT-traced beam."""
import numpy as np
import pytest

from subsecondpbs_b200 import _lib as L
from subsecondpbs_b200 import phantoms

from _parity import assert_stage_parity, oracle_run, run_gpu, stage_report
from test_gpu_parity import _dose_checks

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("index_positions", [True, False])
def test_weq_stage_parity(index_positions):
    case = phantoms.weq_case(index_positions=index_positions)
    eng = run_gpu(case)
    r = oracle_run(case, capture=True, capture_layers=True)
    rep = stage_report(eng, r["capture"])
    assert rep["wepl_max_abs_mm"] == 0.0 and rep["density_max_abs"] == 0.0, rep
    assert rep["wepl_min_max_abs_mm"] == 0.0, rep
    assert_stage_parity(rep)
    _dose_checks(eng.read_dose(), r["dose"], case["dose_resolution"])


def test_weq_beam_in_a_plan_with_ct_beams(hetero_small_case):
    """A WEQ beam and CT-traced beams accumulate into one grid."""
    case = phantoms.weq_case()
    ct_beam = phantoms.rotate_beam(case["beam"], 200.0)
    ct_beam = {k: v for k, v in ct_beam.items()
               if k not in ("water_equivalence", "ray_weq_header", "spot_positions_are_indices")}
    ct_beam["spot_positions"] = np.asarray(hetero_beam_positions(case), np.float32)
    beams = [case["beam"], ct_beam]
    eng = run_gpu(case, beams=beams, keep_debug=False)
    r = oracle_run(case, beams=beams)
    _dose_checks(eng.read_dose(), r["dose"], case["dose_resolution"])


def hetero_beam_positions(case):
    """The weq_case spots back in millimetres."""
    h = case["beam"]["water_equivalence"][:9]
    pos = np.asarray(case["beam"]["spot_positions"], np.float32).reshape(-1, 2)
    return ((pos - 0.5) * np.array([h[7], h[4]]) + np.array([h[6], h[3]])).reshape(-1)


def test_weq_payload_shorter_than_header_is_refused():
    case = phantoms.weq_case()
    beam = dict(case["beam"])
    beam["water_equivalence"] = beam["water_equivalence"][:-5]
    with pytest.raises(L.PbsError) as ex:
        run_gpu(case, beams=[beam], keep_debug=False)
    assert ex.value.code == L.PBS_ERR_GEOMETRY
    assert "smaller than header" in str(ex.value)
