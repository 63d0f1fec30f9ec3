"""The oracle against outputs of the reference itself.

tests/golden/*.npz were produced by tests/golden/make_golden.py, which runs the
reference's subsecondWrapper built from its own sources (oracle/ref/build_ref.sh)
on a B200. The reference samples its BEV dose shifted by the beam's first-inside
step, so the oracle runs with compat_bev_z_shift. The reference samples the CT,
LUTs, CIDD table and BEV dose through the texture unit (8-bit interpolation
weights) with -use_fast_math; the oracle uses exact weights in double precision.
Tolerances per case are the pinned agreement: max |dose - reference| over voxels
above 10 % of Dmax, the 1 %/1 mm gamma pass rate, and the batched radius lists
the reference prints (complete_superposition.cu:476-495), which must be identical
up to single tiles that sit on a bucket boundary. The nuclear-halo case was made by
the reference built with NUCLEAR_CORR=GAUSS_FIT; its halo batched lists
(complete_superposition.cu:660-669) are pinned the same way. The WEQ case drives
the beam with an imported water-equivalence volume and rayweq texel spot
coordinates (the CarbonPBS contract). The *_rt cases run the reference on its own
lookup tables (tables/ as read by its energyReader, tests/golden/reference_tables.npz).

In the rotated cases the body surface crosses the dose voxels obliquely. The first
step of a ray inside the body holds the IDD of a step whose WEPL increment and mass
are sampled from partly filled CT voxels, which can exceed the plateau several
times over (both in the reference and in the oracle); which dose voxel picks up
such a step flips under float rounding of the BEV coordinates. Those cases drop a
pinned number of their largest voxel differences (all on the entrance surface)
before the max-error check; the gamma pass rate still covers every voxel."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

from _parity import gamma_pass_rate, max_rel_err

GOLDEN = Path(__file__).resolve().parent / "golden"

# case -> (max err / Dmax, min gamma pass rate, max tiles that may change bucket,
#          largest voxel differences dropped before the max-error check)
PINS = {
    "water_small": (5e-4, 1.0, 0, 0),
    "water_config1": (5e-4, 1.0, 0, 0),
    "hetero_small": (5e-3, 0.999, 1, 0),
    "hetero_legacy": (2e-2, 0.999, 0, 0),
    "hetero_rot30": (5e-2, 0.998, 0, 0),
    "halo_small": (5e-3, 0.999, 1, 0),
    "weq_small": (5e-4, 1.0, 0, 0),
    "carbon_halo_small": (2e-2, 0.999, 3, 0),
    # The reference's own tables.
    "water_config1_rt": (5e-4, 1.0, 0, 0),
    "hetero_small_rt": (5e-3, 0.999, 1, 0),
    "hetero_mid_rt": (2e-2, 0.999, 1, 0),
    "hetero_rot30_rt": (5e-2, 0.998, 1, 10),
    "halo_small_rt": (5e-3, 0.999, 1, 0),
    "profile_small_rt": (5e-4, 1.0, 1, 0),
    "profile_energy_rows_rt": (5e-4, 1.0, 1, 0),
    "headline_rt": (1e-2, 0.999, 1, 6),
}


def pinned_err(dose, ref, drop):
    """max |dose - ref| / Dmax over voxels above 10 % of Dmax after dropping the
    `drop` largest differences."""
    ref = np.asarray(ref, np.float64)
    m = float(ref.max())
    diff = np.sort(np.abs(np.asarray(dose, np.float64) - ref)[ref > 0.1 * m])[::-1]
    return float(diff[drop] / m) if diff.size > drop else 0.0


def nuclear_model_of(meta):
    """GAUSS_FIT (2) for the cases the reference ran with its nuclear halo, else None."""
    tf = meta.get("transform") or {}
    return {"SOUKUP": 0, "FLUKA": 1, "GAUSS_FIT": 2}[tf["nuclear"]] if "nuclear" in tf else None


def carbon_profile_of(meta):
    """Both profile switches (3) for the cases the reference ran with its CarbonPBS
    lateral profile model on, else 0."""
    return 3 if "profile" in (meta.get("transform") or {}) else 0


def load_case(name):
    import sys

    sys.path.insert(0, str(GOLDEN))
    from make_golden import build_case

    z = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(str(z["meta"]))
    case, beam = build_case(name)
    return z, meta, case, beam


@pytest.mark.parametrize("name", sorted(PINS))
def test_oracle_matches_reference_outputs(name):
    z, meta, case, beam = load_case(name)
    tol, gmin, flips, drop = PINS[name]
    nuc = nuclear_model_of(meta)
    r = O.dose(case, beams=[beam], compat_bev_z_shift=True, capture=True,
               nuclear_model=-1 if nuc is None else nuc, carbon_profile=carbon_profile_of(meta))
    ref = z["dose"].astype(np.float64)
    assert abs(float(ref.max()) - meta["dose_max"]) <= 1e-6 * meta["dose_max"]
    err = pinned_err(r["dose"], ref, drop)
    gp = gamma_pass_rate(r["dose"], ref, case["dose_resolution"])
    assert err < tol, err
    assert gp >= gmin, gp
    ob = r["capture"]["batched"]
    rb = z["batched"]
    assert ob.shape[0] == rb.shape[0]
    moved = int(np.abs(ob - rb).sum()) // 2
    assert moved <= flips, (ob.tolist(), rb.tolist())
    if nuc is not None:
        on, rn = r["capture"]["nuc_batched"], z["nuc_batched"]
        assert on.shape == rn.shape
        assert int(np.abs(on - rn).sum()) // 2 <= flips, (on.tolist(), rn.tolist())


def test_halo_is_what_the_reference_adds():
    """The halo case differs from the same beam without the halo by far more than
    its pinned tolerance: the halo branch itself is pinned."""
    z, meta, case, beam = load_case("halo_small")
    ref = z["dose"].astype(np.float64)
    d = O.dose(case, beams=[beam], compat_bev_z_shift=True)["dose"]
    assert max_rel_err(d, ref) > 0.05


def test_bev_shift_is_what_the_reference_does():
    """Without the reference's BEV depth shift the oracle's Bragg peak sits one
    first-inside step shallower than the reference's."""
    z, meta, case, beam = load_case("water_config1")
    ref = z["dose"].astype(np.float64)
    d = O.dose(case, beams=[beam])["dose"]
    cax_ref = ref[:, 32, 32]
    cax = d[:, 32, 32]
    assert int(np.argmax(cax_ref)) - int(np.argmax(cax)) == 1
    assert max_rel_err(d, ref) > 0.1
