"""The oracle's CarbonPBS lateral profile model (raytracedicom_wrapper.cu:2080-2187,
table shape and per-layer rows at 2816-2862 and 4577-4606) on properties the model
must have: off unless switched on, the overall weight scales the dose linearly, a
beam without a usable table is left alone, and the sigma override widens the
lateral spread as its sigmas grow."""
import numpy as np
import pytest

from oracle import oracle as O
from subsecondpbs_b200 import phantoms
from subsecondpbs_b200.precision import max_rel_err


@pytest.fixture(scope="module")
def case():
    return phantoms.heterogeneous_case(dims=(64, 64, 48), n_layers=3, target_radius_mm=14.0, e_range=(80.0, 120.0))


def _with_weight(beam, value):
    b = dict(beam)
    prof = np.asarray(b["profile_data"], np.float32).reshape(3, -1, 5).copy()
    prof[:, :, 4] = value
    b["profile_data"] = prof.reshape(-1)
    return b


def test_off_by_default_and_without_a_table(case):
    beam = phantoms.with_carbon_profile(case["beam"])
    plain = O.dose(case)["dose"]
    assert np.array_equal(O.dose(case, beams=[beam])["dose"], plain)
    # A table whose shape cannot be inferred (one value short) is not applied.
    short = dict(beam)
    short["profile_data"] = np.asarray(beam["profile_data"], np.float32)[:-1]
    assert np.array_equal(O.dose(case, beams=[short], carbon_profile=3)["dose"], plain)


def test_overall_weight_scales_the_dose(case):
    beam = phantoms.with_carbon_profile(case["beam"])
    plain = O.dose(case)["dose"]
    one = O.dose(case, beams=[_with_weight(beam, 1.0)], carbon_profile=2)["dose"]
    assert max_rel_err(one, plain, thr=0.0) < 1e-12
    half = O.dose(case, beams=[_with_weight(beam, 0.5)], carbon_profile=2)["dose"]
    np.testing.assert_allclose(half, 0.5 * plain, rtol=1e-9, atol=1e-12 * plain.max())
    # A negative weight is clamped to zero (applyCarbonProfileOverallWeightKernel).
    assert not O.dose(case, beams=[_with_weight(beam, -1.0)], carbon_profile=2)["dose"].any()


def test_sigma_override_widens_with_the_profile_sigmas(case):
    beam = phantoms.with_carbon_profile(case["beam"])
    wide = dict(beam)
    prof = np.asarray(beam["profile_data"], np.float32).reshape(3, -1, 5).copy()
    prof[:, :, 2:4] *= 2.0
    wide["profile_data"] = prof.reshape(-1)
    a = O.dose(case, beams=[beam], carbon_profile=1)["dose"]
    b = O.dose(case, beams=[wide], carbon_profile=1)["dose"]
    # Same integral dose spread wider: a lower maximum.
    assert b.max() < 0.97 * a.max()
    assert abs(b.sum() / a.sum() - 1.0) < 0.05
