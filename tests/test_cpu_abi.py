"""The C-ABI library loads without a GPU, exports every declared entry point and
reports validation errors as status codes."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from subsecondpbs_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def _declared_symbols():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = "\n".join(ln for ln in text.splitlines() if not ln.lstrip().startswith("#"))
        names |= set(re.findall(r"(?:PBS_API|RTD_API)\s+[\w\s\*]*?\b(\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _declared_symbols()
    assert {"pbs_subsecond_wrapper", "subsecondWrapper", "pbs_context_add_beam", "pbs_plan_beam"} <= declared
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, f"symbols declared in include/*.h but not exported: {missing}"


def test_version_and_device_count_without_gpu():
    lib = _lib.load()
    assert b"sm_100a" in lib.pbs_version()
    n = C.c_int(-1)
    rc = lib.pbs_device_count(C.byref(n))
    assert rc in (_lib.PBS_OK, _lib.PBS_ERR_CUDA)
    assert n.value >= 0


def test_plan_rejects_invalid_beam(water_case):
    from subsecondpbs_b200.cudaCalDoseRTD import plan_beam

    c = water_case
    bad = dict(c["beam"])
    bad["spot_weights"] = np.ones(3, np.float32)  # does not match summed layer_spot_counts
    with pytest.raises(_lib.PbsError) as e:
        plan_beam(bad, c["energy"], c["ct_dims"], c["ct_resolution"], c["ct_corner"], c["dose_dims"],
                  c["dose_resolution"], c["dose_corner"])
    assert e.value.code == _lib.PBS_ERR_INVALID_ARGUMENT
    assert "spotWeights" in str(e.value)


def test_plan_rejects_bad_grids(water_case):
    from subsecondpbs_b200.cudaCalDoseRTD import plan_beam

    c = water_case
    with pytest.raises(_lib.PbsError) as e:
        plan_beam(c["beam"], c["energy"], (0, 64, 128), c["ct_resolution"], c["ct_corner"], c["dose_dims"],
                  c["dose_resolution"], c["dose_corner"])
    assert e.value.code == _lib.PBS_ERR_INVALID_ARGUMENT
    with pytest.raises(_lib.PbsError):
        plan_beam(c["beam"], c["energy"], c["ct_dims"], (2.0, -1.0, 2.0), c["ct_corner"], c["dose_dims"],
                  c["dose_resolution"], c["dose_corner"])


def test_plan_requires_ray_spacing_in_legacy_mode(water_case):
    from subsecondpbs_b200.cudaCalDoseRTD import plan_beam

    c = water_case
    b = {k: v for k, v in c["beam"].items() if k not in ("layer_spot_counts", "spot_positions", "spot_weights")}
    b["ray_spacing"] = (0.0, 0.0)
    with pytest.raises(_lib.PbsError) as e:
        plan_beam(b, c["energy"], c["ct_dims"], c["ct_resolution"], c["ct_corner"], c["dose_dims"],
                  c["dose_resolution"], c["dose_corner"])
    assert e.value.code == _lib.PBS_ERR_GEOMETRY


def test_struct_layouts_match_header():
    # Field counts of the ctypes mirrors equal the members declared in the header.
    text = (ROOT / "include" / "subsecondpbs.h").read_text()

    def members(struct):
        body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (struct, struct), text, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        n = 0
        for decl in body.split(";"):
            decl = decl.strip()
            if decl:
                n += 1
        return n

    assert members("PbsBeamDesc") == len(_lib.PbsBeamDesc._fields_)
    assert members("PbsEnergyDesc") == len(_lib.PbsEnergyDesc._fields_)
    assert members("PbsBeamStats") == len(_lib.PbsBeamStats._fields_)
    assert members("PbsLayerStats") == len(_lib.PbsLayerStats._fields_)


def test_server_stats_layout_matches_header():
    text = (ROOT / "include" / "subsecondpbs.h").read_text()
    body = re.search(r"typedef struct PbsServerStats \{(.*?)\} PbsServerStats;", text, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if decl:
            assert decl.startswith("long long ")
            names += [n.strip() for n in decl[len("long long "):].split(",")]
    assert names == [n for n, _ in _lib.PbsServerStats._fields_]


def test_server_refuses_to_start_without_a_device():
    """No GPU here: creating a server fails with a status, not a crash."""
    lib = _lib.load()
    h = C.c_void_p()
    n = C.c_int(0)
    lib.pbs_device_count(C.byref(n))
    if n.value > 0:
        pytest.skip("a GPU is visible")
    rc = lib.pbs_server_create(0, 2, 0, C.byref(h))
    assert rc != _lib.PBS_OK and not h.value
    assert lib.pbs_server_destroy(None) == _lib.PBS_OK
    assert lib.pbs_server_submit(None, 0, 0, None, 0, 0, None) == _lib.PBS_ERR_INVALID_ARGUMENT
