"""The plain data layouts of include/pbs_layouts.h against the reference's own
structs (include/core/common.cuh:39-228).

tests/golden/reference_layouts.json holds each struct's size and member offsets as
measured by compiling against the reference's header (tests/golden/make_layouts.py).
The mirrors are measured here by compiling the same program against
include/pbs_layouts.h, as C and as C++. Where a reference checkout is present
($REFERENCE_DIR, else <repo>/../reference) the reference is measured again."""
import json
import os
import shutil
import sys
from pathlib import Path

import numpy as np
import pytest

from subsecondpbs_b200 import doseio

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
CHECKOUT = Path(os.environ.get("REFERENCE_DIR", str(ROOT.parent / "reference")))
sys.path.insert(0, str(GOLDEN))
from make_layouts import measure, program, reference_layouts  # noqa: E402

MIRROR_NAMES = {
    "vec3f": "PbsVec3f", "vec3i": "PbsVec3i", "vec2f": "PbsVec2f", "Grid": "PbsGrid", "Source": "PbsSource",
    "Beam": "PbsBeam", "SubspotInfo": "PbsSubspotInfo", "CPBGrid": "PbsCPBGrid",
    ("Grid", "upperCorner"): "upper_corner",
    ("Source", "sourcePos"): "source_pos", ("Source", "isoPos"): "iso_pos", ("Source", "vsDirX"): "vs_dir_x",
    ("Source", "vSAD"): "v_sad",
    ("Beam", "transCutoff"): "trans_cutoff", ("Beam", "longitudalCutoff"): "longitudal_cutoff",
    ("Beam", "eneIdx"): "ene_idx",
    ("SubspotInfo", "deltaX"): "delta_x", ("SubspotInfo", "deltaY"): "delta_y", ("SubspotInfo", "sigmaX"): "sigma_x",
    ("SubspotInfo", "sigmaY"): "sigma_y", ("SubspotInfo", "eneIdx"): "ene_idx",
    ("SubspotInfo", "effectiveSigma"): "effective_sigma", ("SubspotInfo", "isValid"): "is_valid",
    ("CPBGrid", "nLayers"): "n_layers",
}


def golden():
    return json.loads((GOLDEN / "reference_layouts.json").read_text())["layouts"]


@pytest.mark.parametrize("lang", ["c", "c++"])
def test_mirrors_match_the_reference_layouts(lang):
    inc = f'#include "{ROOT / "include" / "pbs_layouts.h"}"'
    src = program(inc, MIRROR_NAMES)
    cc = shutil.which("gcc" if lang == "c" else "g++")
    got = measure(src, [cc, "-x", lang, "-std=c11" if lang == "c" else "-std=c++17"], ".c" if lang == "c" else ".cpp")
    assert got == golden()


def test_reference_names_alias_the_mirrors():
    inc = f'#define PBS_REFERENCE_NAMES\n#include "{ROOT / "include" / "pbs_layouts.h"}"'
    names = {k: v for k, v in MIRROR_NAMES.items() if isinstance(k, tuple)}
    got = measure(program(inc, names), [shutil.which("gcc"), "-x", "c", "-std=c11"], ".c")
    assert got == golden()


@pytest.mark.skipif(not (CHECKOUT / "include" / "core" / "common.cuh").exists(), reason="no reference checkout")
def test_golden_is_the_reference_header():
    assert reference_layouts(CHECKOUT) == golden()


def test_dose_bin_round_trip(tmp_path):
    rng = np.random.Generator(np.random.PCG64(3))
    dose = rng.random((5, 4, 3), dtype=np.float32)
    p = tmp_path / "dose.bin"
    doseio.write_dose_bin(p, dose, (2.0, 2.0, 2.5), (-10.0, -8.0, 0.5))
    raw = p.read_bytes()
    assert len(raw) == 36 + dose.nbytes
    assert np.frombuffer(raw[:12], "<i4").tolist() == [3, 4, 5]
    back, sp, org = doseio.read_dose_bin(p)
    assert np.array_equal(back, dose) and sp == (2.0, 2.0, 2.5) and org == (-10.0, -8.0, 0.5)
    p.write_bytes(raw[:-4])
    with pytest.raises(ValueError):
        doseio.read_dose_bin(p)
