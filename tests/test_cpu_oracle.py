"""Properties of the CPU oracle itself: physical invariants of the reference model
(Bragg-peak depth, linearity in spot weights, symmetry, energy bookkeeping) and
known answers of the integer radius / batching rules."""
import numpy as np
import pytest

from oracle import oracle as O
from subsecondpbs_b200 import phantoms


def test_water_bragg_peak_depth_matches_lut(water_case):
    r = O.dose(water_case, capture=True)
    d = r["dose"]
    cax = d[:, d.shape[1] // 2, d.shape[2] // 2]
    # The beam enters at z index 0 (travelling +z); voxel k is centred 2k mm deep.
    depth = 2.0 * float(np.argmax(cax))
    peak = float(r["capture"]["plan"]["layer_params"][0][2])
    assert abs(depth - peak) <= 2.0, (depth, peak)


def test_bev_shift_compat_moves_dose_by_first_inside(water_case):
    a = O.dose(water_case)["dose"]
    b = O.dose(water_case, compat_bev_z_shift=True)["dose"]
    ca = a[:, 32, 32]
    cb = b[:, 32, 32]
    # The reference samples BEV planes shifted by the beam's first-inside step (1 here):
    # its Bragg peak appears one 2 mm step deeper.
    assert int(np.argmax(cb)) - int(np.argmax(ca)) == 1


def test_linearity_in_spot_weights(hetero_small_case):
    c = hetero_small_case
    d1 = O.dose(c)["dose"]
    b2 = dict(c["beam"])
    b2["spot_weights"] = np.asarray(b2["spot_weights"], np.float32) * 2.0
    d2 = O.dose(c, beams=[b2])["dose"]
    # Exact up to the IDD stage's live-ray threshold (ray weight < 1e-6 is dead,
    # idd_sigma.cu:78), which only moves sub-1e-5 Dmax dose at the field edge.
    np.testing.assert_allclose(d2, 2.0 * d1, rtol=1e-6, atol=1e-5 * d1.max())


def test_additivity_over_spot_subsets(hetero_small_case):
    c = hetero_small_case
    w = np.asarray(c["beam"]["spot_weights"], np.float32)
    ba, bb = dict(c["beam"]), dict(c["beam"])
    mask = np.arange(w.size) % 2 == 0
    # Keep every weight above the 1e-6 live-ray threshold of the IDD stage by
    # splitting weights instead of zeroing spots.
    ba["spot_weights"] = np.where(mask, 0.25 * w, 0.75 * w).astype(np.float32)
    bb["spot_weights"] = np.where(mask, 0.75 * w, 0.25 * w).astype(np.float32)
    d = O.dose(c)["dose"]
    dab = O.dose(c, beams=[ba])["dose"] + O.dose(c, beams=[bb])["dose"]
    np.testing.assert_allclose(dab, d, rtol=1e-6, atol=1e-5 * d.max())


def test_lateral_symmetry_water():
    c = phantoms.water_phantom_case(dims=(64, 64, 96))
    d = O.dose(c)["dose"]
    m = d.max()
    # Spots are symmetric about the beam axis through voxel centre (31.5, 31.5):
    # mirror images differ only by the lattice half-cell and interpolation.
    sym = np.abs(d - d[:, ::-1, ::-1]).max() / m
    assert sym < 0.05


def test_multi_beam_accumulates(hetero_small_case):
    c = hetero_small_case
    b0 = phantoms.rotate_beam(c["beam"], 0.0)
    b1 = phantoms.rotate_beam(c["beam"], 120.0)
    d0 = O.dose(c, beams=[b0])["dose"]
    d1 = O.dose(c, beams=[b1])["dose"]
    both = O.dose(c, beams=[b0, b1])["dose"]
    np.testing.assert_allclose(both, d0 + d1, rtol=1e-9, atol=1e-15)


def test_initial_dose_is_accumulated_into(water_case):
    base = np.full((128, 64, 64), 1e-9)
    d0 = O.dose(water_case)["dose"]
    d1 = O.dose(water_case, initial=base)["dose"]
    np.testing.assert_allclose(d1, d0 + base, rtol=1e-12, atol=1e-20)


@pytest.mark.parametrize("m,expected", [
    (float("inf"), 0),       # dead tile
    (3.0, 1),                # 3/(sqrt2*3)+0.5 = 1.207
    (0.3, 7),                # 7.57
    (0.0655, 32),            # 32.88 -> 32
    (0.0640, 33),            # 33.64 -> overflow bucket
    (1e-30, 33),
])
def test_radius_bucket_known_answers(m, expected):
    assert O.radius_bucket(m) == expected


def test_batching_known_answers():
    # complete_superposition.cu:476-483: walk down from the largest radius, merging
    # buckets until a batch holds at least 16 tiles.
    h = np.zeros(34, np.int32)
    h[0], h[1], h[2], h[3], h[5], h[9] = 100, 4, 20, 3, 10, 2
    b, m = O.batch(h)
    # rad 9 (2) opens batch 9; rad 8..6 add 0; rad 5 (10) -> 12; rad 4 -> 12; rad 3 -> 15; rad 2 -> 35 >= 16
    # closes, next batch opens at 1: rad 1 adds 4.
    assert b[9] == 2 + 10 + 3 + 20 and b[1] == 4 and b[0] == 100
    assert list(m[1:10]) == [1, 9, 9, 9, 9, 9, 9, 9, 9]
    h2 = np.zeros(34, np.int32)
    h2[33], h2[32], h2[10] = 5, 20, 40
    b2, m2 = O.batch(h2)
    # Primary overflow is merged into radius 32 before batching. The batch opened at
    # radius 31 after closing 32 stays open across the empty buckets, so the
    # radius-10 tiles are superposed with radius 31 (the reference's walk does this).
    assert b2[32] == 25 and b2[31] == 40 and b2[10] == 0
    assert m2[33] == 32 and m2[10] == 31


def test_oracle_radius_matches_product_formula():
    # Bucket formula evaluated in single precision exactly as the CUDA kernel does.
    rng = np.random.default_rng(7)
    for m in rng.uniform(0.05, 5.0, 2000).astype(np.float32):
        q = np.float32(np.float32(3.0) / (np.float32(1.41421354) * m)) + np.float32(0.5)
        exp = 33 if q >= 34 else min(int(q), 33)
        assert O.radius_bucket(float(m)) == exp
