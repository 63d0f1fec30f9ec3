"""Biological maps on the GPU (pbs_context_set_bio_model / read_bio_map) against
the oracle on identical seeded inputs: the CarbonPBS LQ and MKM RBE maps
(carbonPBS/deviceCalDose.cu:587-772, 1060-1126) on the pencil-beam dose, with the
dose channel, dose-averaged LET, mixed parameters and RBE within the path's
tolerance; the accumulators restart with a dose reset; halo beams are refused."""
import numpy as np
import pytest

from oracle import oracle as O
from subsecondpbs_b200 import _lib, phantoms
from subsecondpbs_b200.precision import max_rel_err

from _parity import DOSE_TOL_FRAC_DMAX

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scaled_case(hetero_small_case):
    c = hetero_small_case
    d = O.dose(c)["dose"]
    beam = dict(c["beam"])
    beam["spot_weights"] = np.asarray(beam["spot_weights"], np.float32) * np.float32(2.0 / d.max())
    return dict(c, beam=beam)


def _engine(case, bio):
    from subsecondpbs_b200.cudaCalDoseRTD import DoseEngine

    eng = DoseEngine(0)
    eng.set_energy(case["energy"])
    eng.set_ct(case["ct"], case["ct_dims"], case["ct_resolution"], case["ct_corner"])
    eng.set_dose_grid(case["dose_dims"], case["dose_resolution"], case["dose_corner"])
    eng.set_bio_model(bio)
    return eng


@pytest.mark.parametrize("model", ["lq", "mkm"])
def test_bio_maps_match_the_oracle(scaled_case, model):
    bio = phantoms.bio_model(model)
    eng = _engine(scaled_case, bio)
    eng.reset_dose()
    eng.add_beam(scaled_case["beam"])
    r = O.dose(scaled_case, bio=bio)
    dose = r["dose"]
    hot = dose > 0.1 * dose.max()
    assert max_rel_err(eng.read_bio_map("dose"), dose) < 1e-4
    assert max_rel_err(eng.read_dose(), dose) < 1e-4
    names = ["letd", "rbe", "rbe_dose"] + (["alpha", "beta"] if model == "lq" else ["z1d"])
    for name in names:
        got = eng.read_bio_map(name).astype(np.float64)
        want = O.bio_map(bio, r["bio_acc"], name)
        rel = np.abs(got - want)[hot] / np.maximum(np.abs(want[hot]), 1e-30)
        assert float(rel.max()) < DOSE_TOL_FRAC_DMAX, (name, float(rel.max()))
    eng.close()


def test_reset_restarts_the_accumulators(scaled_case):
    bio = phantoms.bio_model("lq")
    eng = _engine(scaled_case, bio)
    eng.add_beam(scaled_case["beam"])
    eng.add_beam(scaled_case["beam"])
    two = eng.read_bio_map("dose")
    eng.reset_dose()
    eng.add_beam(scaled_case["beam"])
    one = eng.read_bio_map("dose")
    assert max_rel_err(two, 2.0 * one) < 1e-5
    # The RBE of twice the same beam differs from one beam's (the LQ dose response).
    eng.close()


def test_halo_beams_are_refused_while_a_model_is_set(scaled_case):
    from subsecondpbs_b200 import tables

    case = dict(scaled_case, energy=tables.synthetic_nuclear_tables(scaled_case["energy"]))
    eng = _engine(case, phantoms.bio_model("lq"))
    with pytest.raises(_lib.PbsError) as e:
        eng.add_beam(case["beam"], nuclear_correction=True)
    assert e.value.code == _lib.PBS_ERR_UNSUPPORTED
    eng.set_bio_model(None)
    eng.add_beam(case["beam"], nuclear_correction=True)
    eng.close()
