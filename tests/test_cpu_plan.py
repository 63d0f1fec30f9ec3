"""Host beam planning of the library against the oracle's restatement: every
integer decision and every single-precision geometry value must be identical."""
import numpy as np
import pytest

from oracle import oracle as O
from subsecondpbs_b200 import phantoms
from subsecondpbs_b200.cudaCalDoseRTD import plan_beam


def _both(case, beam=None):
    beam = beam if beam is not None else case["beam"]
    p = plan_beam(beam, case["energy"], case["ct_dims"], case["ct_resolution"], case["ct_corner"],
                  case["dose_dims"], case["dose_resolution"], case["dose_corner"], with_lattice=True)
    o = O.plan(case, beam, with_lattice=True)
    return p, o


def _compare(p, o):
    assert p["num_layers"] == o["num_layers"]
    assert p["conv_mode"] == o["conv_mode"]
    assert list(p["ray_dims"]) == [o["ray_x"], o["ray_y"]]
    assert list(p["superp_dims"]) == [o["pitch_x"], o["pitch_y"]]
    assert p["tracer_steps"] == o["steps"]
    if p["conv_mode"] == 0:
        assert list(p["lattice_dims"]) == [o["lat_nx"], o["lat_ny"]]
        assert list(p["lattice_delta"]) == [o["lat_dx"], o["lat_dy"]]
        assert list(p["lattice_offset"]) == [o["lat_ox"], o["lat_oy"]]
        np.testing.assert_array_equal(p["lattice"], o["lattice"])
    assert list(p["cpb_corner"]) == list(o["cpb_corner"])
    assert list(p["cpb_resolution"]) == list(o["cpb_res"])
    assert list(p["fan_corner"]) == list(o["fan_corner"])
    assert list(p["fan_delta"]) == list(o["fan_delta"])
    assert list(p["source_dist"]) == list(o["source_dist"])
    assert p["len_to_mm"] == o["len_to_mm"]
    assert p["energy_depth_to_mm"] == o["energy_depth_to_mm"]
    assert p["max_peak_depth_mm"] == o["max_peak_depth_mm"]
    np.testing.assert_array_equal(p["layer_params"], o["layer_params"])


def test_plan_water_phantom(water_case):
    p, o = _both(water_case)
    _compare(p, o)
    assert list(p["ray_dims"]) == [96, 80] and p["tracer_steps"] == 128


def test_plan_heterogeneous_headline(hetero_case):
    p, o = _both(hetero_case)
    _compare(p, o)
    # 5 mm hexagonal lattice: 2.5 mm x 4.33 mm half-empty raw lattice.
    assert list(p["lattice_dims"]) == [25, 15]
    assert list(p["ray_dims"]) == [128, 104]


@pytest.mark.parametrize("angle", [0.0, 120.0, 240.0, 33.0])
def test_plan_rotated_gantry(hetero_small_case, angle):
    beam = phantoms.rotate_beam(hetero_small_case["beam"], angle)
    p, o = _both(hetero_small_case, beam)
    _compare(p, o)


def test_plan_legacy_cpb_mode(hetero_small_case):
    beam = phantoms.legacy_beam(hetero_small_case["beam"])
    p, o = _both(hetero_small_case, beam)
    assert p["conv_mode"] == 1
    _compare(p, o)


def test_plan_centimetre_units():
    case = phantoms.water_phantom_case(dims=(32, 32, 48), res=(2.0, 2.0, 2.0))
    case = phantoms.to_centimetres(case)
    p, o = _both(case)
    _compare(p, o)
    assert p["len_to_mm"] == 10.0


def test_plan_virtual_source_from_spot_directions(hetero_small_case):
    beam = phantoms.with_spot_directions(hetero_small_case["beam"], sad_x=1800.0, sad_y=2300.0)
    p, o = _both(hetero_small_case, beam)
    _compare(p, o)
    assert abs(p["source_dist"][0] - 1800.0) < 5.0 and abs(p["source_dist"][1] - 2300.0) < 5.0


def test_plan_single_column_lattice(water_case):
    beam = dict(water_case["beam"])
    pos = np.asarray(beam["spot_positions"], np.float32).reshape(-1, 2).copy()
    pos[:, 0] = 0.0
    beam["spot_positions"] = pos.reshape(-1)
    p, o = _both(water_case, beam)
    _compare(p, o)
    # A single x column keeps the reference's sentinel step of 1e20.
    assert p["lattice_dims"][0] == 1 and p["lattice_delta"][0] == np.float32(1e20)


def test_plan_descending_and_out_of_range_energies(water_case):
    case = dict(water_case)
    e = dict(case["energy"])
    for k in ("energies_per_u", "peak_depths", "scale_facts"):
        e[k] = np.ascontiguousarray(np.asarray(e[k])[::-1])
    e["cidd_matrix"] = np.ascontiguousarray(np.asarray(e["cidd_matrix"])[::-1])
    case["energy"] = e
    for energy in (150.0, 30.0, 400.0, float(e["energies_per_u"][5])):
        beam = dict(case["beam"])
        beam["energies"] = np.array([energy], np.float32)
        p, o = _both(case, beam)
        _compare(p, o)
