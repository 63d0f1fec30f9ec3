"""The reference's own lookup tables: the parser against the reference's parser, the
table fixture, and what the tables put into the dose.

tests/golden/reference_tables.npz holds the reference's tables/ files as read by
the reference's energyReader (src/utils/energy_reader.cpp:21-185; made by
tests/golden/make_tables.py). Where a reference checkout is present
($REFERENCE_DIR, else <repo>/../reference) the package's parser is run on its text
files and must give the same float32 bits; where the reference library built by
oracle/ref/build_ref.sh is present as well, its energyReader is run again here."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from subsecondpbs_b200 import phantoms, tables

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
FIXTURE = GOLDEN / "reference_tables.npz"
CHECKOUT = Path(os.environ.get("REFERENCE_DIR", str(ROOT.parent / "reference")))
REF_TABLES = CHECKOUT / "tables"
REF_NUC_LIB = ROOT / "oracle" / "_ref" / "librtd_nuc.so"

sys.path.insert(0, str(GOLDEN))
from make_tables import reference_energy_reader, same_tables  # noqa: E402

needs_checkout = pytest.mark.skipif(not (REF_TABLES / tables.PROTON_FILE).exists(),
                                    reason="no reference checkout with tables/")


@pytest.fixture(scope="module")
def fixture_tables():
    return tables.load_table_npz(FIXTURE)


def test_fixture_layout(fixture_tables):
    t = fixture_tables
    ne, ns = t["n_energies"], t["n_energy_samples"]
    assert (ne, ns) == (147, 1024)
    assert t["cidd_matrix"].shape == (ne, ns) and t["cidd_matrix"].dtype == np.float32
    assert np.all(np.diff(t["energies_per_u"]) > 0) and np.all(np.diff(t["peak_depths"]) > 0)
    # Every CIDD row is cumulative: non-decreasing along depth.
    assert np.all(np.diff(t["cidd_matrix"], axis=1) >= 0)
    for key, scale in (("density", 1.0), ("sp", 1.0), ("rrl", 1000.0)):
        assert t[f"n_{key}_samples"] == 3072 and t[f"{key}_vector"].shape == (3072,)
        assert t[f"{key}_scale_fact"] == scale
    assert t["nuc_weight_matrix"].shape == (ne, ns) and t["nuc_sq_sigma_matrix"].shape == (ne, ns)


def test_peak_depths_are_the_reference_expectations(fixture_tables):
    """The reference's water-phantom test names the Bragg-peak depths of these tables:
    103.75 mm at 120 MeV, 173.92 mm at 160 MeV, 214.05 mm at 180 MeV
    (src/tests/wrapper_integration_test.cu:3529)."""
    t = fixture_tables
    for e, depth in ((120.0, 103.75), (160.0, 173.92), (180.0, 214.05)):
        assert abs(np.interp(e, t["energies_per_u"], t["peak_depths"]) - depth) < 0.01


@needs_checkout
def test_parser_is_bit_identical_to_the_fixture(fixture_tables):
    mine = tables.energy_reader(REF_TABLES, nuclear=True)
    assert same_tables(mine, fixture_tables) == []


@needs_checkout
@pytest.mark.skipif(not REF_NUC_LIB.exists(), reason="reference library not built (oracle/ref/build_ref.sh GAUSS_FIT)")
def test_reference_energy_reader_gives_the_fixture(fixture_tables):
    ref = reference_energy_reader(REF_TABLES, REF_NUC_LIB)
    assert same_tables(ref, fixture_tables) == []


@needs_checkout
@pytest.mark.parametrize("model", sorted(tables.NUCLEAR_FILES))
def test_every_nuclear_table_parses_on_the_proton_axes(model):
    t = tables.energy_reader(REF_TABLES, nuclear=True, nuclear_file=tables.NUCLEAR_FILES[model])
    w, s2 = t["nuc_weight_matrix"], t["nuc_sq_sigma_matrix"]
    assert w.shape == s2.shape == t["cidd_matrix"].shape
    assert np.all(np.isfinite(w)) and np.all(np.isfinite(s2))
    # The fit table holds one slightly negative weight (-0.0063 at 216.6 MeV, depth 0).
    assert np.all(w > -0.01) and np.all(w < 1) and np.all(s2 >= 0)


def test_nuclear_header_mismatch_is_refused(tmp_path, fixture_tables):
    t = dict(fixture_tables)
    tables.write_tables(tmp_path, t)
    text = (tmp_path / tables.NUCLEAR_FILE).read_text().split("\n")
    energies = text[2].split()
    energies[5] = str(float(energies[5]) + 0.5)
    text[2] = " ".join(energies)
    (tmp_path / tables.NUCLEAR_FILE).write_text("\n".join(text))
    with pytest.raises(ValueError, match="energies differ"):
        tables.energy_reader(tmp_path, nuclear=True)


def test_text_round_trip_is_bit_exact(tmp_path, fixture_tables):
    tables.write_tables(tmp_path, fixture_tables)
    back = tables.energy_reader(tmp_path, nuclear=True)
    assert same_tables(back, fixture_tables) == []


@pytest.mark.parametrize("energy_mev", [120.0, 160.0, 180.0])
def test_water_bragg_peak_with_the_reference_tables(fixture_tables, energy_mev):
    t = {k: v for k, v in fixture_tables.items() if not k.startswith("nuc")}
    c = phantoms.water_phantom_case(dims=(32, 32, 128), energy_mev=energy_mev, n_side=5, energy=t)
    r = O.dose(c, capture=True)
    cax = r["dose"][:, 16, 16]
    peak = float(r["capture"]["plan"]["layer_params"][0][2])
    # Voxel k is centred 2k mm deep: the peak voxel is within one 2 mm voxel (and the
    # half voxel of the water surface) of the table's peak depth.
    assert abs(2.0 * float(np.argmax(cax)) - peak) <= 2.5
