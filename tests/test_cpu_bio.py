"""The oracle's biological maps (the CarbonPBS LQ and MKM RBE maps,
carbonPBS/deviceCalDose.cu:587-772 and 1060-1126, on the pencil-beam dose):
known answers of the map arithmetic, and the dose-weighted mixing on a model whose
LET is the same everywhere."""
import numpy as np
import pytest

from oracle import oracle as O
from subsecondpbs_b200 import phantoms


@pytest.fixture(scope="module")
def case():
    c = phantoms.heterogeneous_case(dims=(64, 64, 48), n_layers=3, target_radius_mm=14.0, e_range=(80.0, 120.0))
    d = O.dose(c)["dose"]
    # Spot weights scaled so that the maximum dose is 2 (Gy): MKM's RBE depends on it.
    beam = dict(c["beam"])
    beam["spot_weights"] = np.asarray(beam["spot_weights"], np.float32) * np.float32(2.0 / d.max())
    return dict(c, beam=beam)


def _acc(values):
    d, c0, c1, c2 = (np.asarray(v, np.float64).reshape(1, 1, -1) for v in values)
    return np.stack([d, c0, c1, c2])


def test_lq_map_arithmetic():
    """LQRBEKernel: RBE = 3.988565 / D10, D10 the dose of 10 % survival of the mixed
    alpha and beta = (mixed sqrt(beta))^2; 1 where the dose, alpha or beta is 0."""
    bio = phantoms.bio_model("lq")
    d = np.array([2.0, 0.0, 1.0, 3.0])
    a, sb = np.array([0.3, 0.5, 0.0, 0.9]), np.array([0.25, 0.2, 0.2, 0.0])
    acc = _acc([d, a * d, sb * d, 7.0 * d])
    rbe = O.bio_map(bio, acc, "rbe").reshape(-1)
    beta = sb ** 2
    d10 = (-a[0] + np.sqrt(a[0] ** 2 + 4 * 2.302585 * beta[0])) / (2 * beta[0])
    assert rbe[0] == pytest.approx(3.988565 / d10, rel=1e-12)
    assert list(rbe[1:]) == [1.0, 1.0, 1.0]
    assert O.bio_map(bio, acc, "letd").reshape(-1)[0] == pytest.approx(7.0)
    assert O.bio_map(bio, acc, "beta").reshape(-1)[0] == pytest.approx(0.0625)
    assert O.bio_map(bio, acc, "rbe_dose").reshape(-1)[0] == pytest.approx(2.0 * rbe[0])


def test_mkm_map_arithmetic():
    """mkmRBEMapKernel: alpha = 0.172 + beta0 z, photon dose of equal effect over the
    ion dose; 1 at or below 1e-3 Gy."""
    bio = phantoms.bio_model("mkm")
    d = np.array([2.0, 1e-4])
    z = np.array([1.5, 3.0])
    acc = _acc([d, z * d, 0 * d, 0 * d])
    rbe = O.bio_map(bio, acc, "rbe").reshape(-1)
    a = 0.172 + 0.0593 * 1.5
    t2 = 0.3312 / 2 / 0.0593
    want = (-t2 + np.sqrt(t2 ** 2 + (a * 2.0 + 0.0593 * 4.0) / 0.0593)) / 2.0
    # alpha0, beta0 cross the C ABI as float32.
    assert rbe[0] == pytest.approx(want, rel=1e-6) and rbe[1] == 1.0
    assert O.bio_map(bio, acc, "z1d").reshape(-1)[0] == pytest.approx(a, rel=1e-6)


@pytest.mark.parametrize("model", ["lq", "mkm"])
def test_constant_let_mixes_to_constants(case, model):
    bio = phantoms.bio_model(model)
    bio["let_table"] = np.full_like(bio["let_table"], 20.0)
    r = O.dose(case, bio=bio)
    acc = r["bio_acc"]
    dose = r["dose"]
    hot = dose > 0.1 * dose.max()
    np.testing.assert_allclose(acc[0], dose, rtol=0, atol=1e-12 * dose.max())
    assert np.allclose(O.bio_map(bio, acc, "letd")[hot], 20.0, rtol=1e-9)
    li = np.log10(20.0) / 0.01
    if model == "lq":
        want = np.interp(li, np.arange(bio["lq_alpha"].size), bio["lq_alpha"])
        assert np.allclose(O.bio_map(bio, acc, "alpha")[hot], want, rtol=1e-6)
    else:
        want = 0.172 + 0.0593 * np.interp(li, np.arange(bio["z1d"].size), bio["z1d"])
        assert np.allclose(O.bio_map(bio, acc, "z1d")[hot], want, rtol=1e-6)


def test_lq_rbe_rises_with_let(case):
    bio = phantoms.bio_model("lq")
    r = O.dose(case, bio=bio)
    letd = O.bio_map(bio, r["bio_acc"], "letd")
    rbe = O.bio_map(bio, r["bio_acc"], "rbe")
    hot = r["dose"] > 0.1 * r["dose"].max()
    # Voxels of high LET (near the end of range) carry a higher RBE than the entrance.
    lo, hi = np.quantile(letd[hot], [0.1, 0.9])
    assert rbe[hot & (letd >= hi)].mean() > rbe[hot & (letd <= lo)].mean()
