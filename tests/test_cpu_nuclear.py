"""Nuclear halo branch of the oracle: contract checks and properties (CPU only)."""
import numpy as np
import pytest

from oracle import oracle as O
from subsecondpbs_b200 import phantoms, tables


def _halo_case(case):
    out = dict(case)
    out["energy"] = tables.synthetic_nuclear_tables(case["energy"])
    return out


def test_halo_contract(hetero_small_case):
    # enforceNuclearCorrectionContract (wrapper.cu:1077-1097) and the raw-lattice
    # requirement (wrapper.cu:3416-3420).
    with pytest.raises(RuntimeError, match="nuclear_weight"):
        O.dose(hetero_small_case, nuclear_model=2)
    case = _halo_case(hetero_small_case)
    with pytest.raises(RuntimeError, match="raw spot lattice"):
        O.dose(case, beams=[phantoms.legacy_beam(case["beam"])], nuclear_model=2)
    unaligned = dict(case)
    unaligned["energy"] = dict(case["energy"], nuclear_tables_aligned_to_primary_axis=False)
    with pytest.raises(RuntimeError, match="aligned"):
        O.dose(unaligned, nuclear_model=2)


def test_halo_plan_maps_every_lattice_cell(hetero_small_case):
    case = _halo_case(hetero_small_case)
    cap = O.dose(case, capture=True, nuclear_model=2)["capture"]
    pl = cap["plan"]
    assert pl["nuc_x"] % 32 == 0 and pl["nuc_y"] % 8 == 0
    assert pl["nuc_x"] >= pl["lat_nx"] and pl["nuc_y"] >= pl["lat_ny"]
    cells = cap["ray_to_nuc"][cap["ray_to_nuc"] >= 0]
    # One ray per lattice cell (ray pitch finer than the lattice), all cells inside the lattice.
    assert cells.size == pl["lat_nx"] * pl["lat_ny"] == np.unique(cells).size
    assert ((cells % pl["nuc_x"]) < pl["lat_nx"]).all() and ((cells // pl["nuc_x"]) < pl["lat_ny"]).all()
    assert cap["nuc_superpose_fma"] > 0 and cap["nuc_bev"].max() > 0


def test_halo_dose_is_linear_in_spot_weights(hetero_small_case):
    case = _halo_case(hetero_small_case)
    b2 = dict(case["beam"])
    b2["spot_weights"] = np.asarray(case["beam"]["spot_weights"], np.float32) * 2.0
    d1 = O.dose(case, nuclear_model=2)["dose"]
    d2 = O.dose(case, beams=[b2], nuclear_model=2)["dose"]
    assert np.abs(d2 - 2.0 * d1).max() < 1e-6 * d2.max()


def test_halo_models_differ(hetero_small_case):
    case = _halo_case(hetero_small_case)
    doses = [O.dose(case, nuclear_model=m)["dose"] for m in (0, 1, 2)]
    base = O.dose(hetero_small_case)["dose"]
    for d in doses:
        assert np.abs(d - base).max() > 1e-3 * base.max()
    assert np.abs(doses[0] - doses[2]).max() > 1e-4 * base.max()
