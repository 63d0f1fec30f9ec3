"""`pbs_operator_batch_plan` (host only, no GPU) against buildRTDOperatorBatchPlan
(include/core/rtd_operator_mode.h:43-111): bit-exact spans and batches on seeded
beams and on every early-return case of the reference's validation, checked
against the CPU restatement (oracle/operator_plan.py) and, where the reference
library built by oracle/ref/build_ref.sh is present, against the reference's own
header compiled into it (ref_operator_batch_plan of oracle/ref/ref_shim.cu)."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from oracle.operator_plan import operator_batch_plan as oracle_plan
from subsecondpbs_b200.operator_mode import operator_batch_plan

SEED = 20261203


def _beam(counts, n_energies=None, weights=None, positions=None, directions=None, cutoffs=True):
    counts = np.asarray(counts, dtype=np.int32)
    total = int(max(counts.sum(), 0))
    b = {"layer_spot_counts": counts,
         "energies": np.linspace(70.0, 180.0, len(counts) if n_energies is None else n_energies, dtype=np.float32)}
    if cutoffs:
        b["layer_longitudinal_cutoffs"] = np.arange(len(counts), dtype=np.float32) * 0.5 + 1.0
    b["spot_weights"] = np.ones(total if weights is None else weights, dtype=np.float32)
    b["spot_positions"] = np.zeros(2 * total if positions is None else positions, dtype=np.float32)
    if directions is not None:
        b["spot_beam_directions"] = np.zeros(directions, dtype=np.float32)
    return b


REF_LIB = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "librtd.so"


def _reference_plan(beam, m):
    """The reference header's plan through the shim, in operator_batch_plan's form."""
    from subsecondpbs_b200 import _lib

    lib = C.CDLL(str(REF_LIB))
    f = lib.ref_operator_batch_plan
    f.restype = C.c_int
    bd, keep = _lib.beam_desc(beam)
    info = (C.c_int * 6)()
    spans = (_lib.PbsOperatorLayerSpan * 4096)()
    batches = (_lib.PbsOperatorBatch * 4096)()
    assert f(C.byref(bd), int(m), spans, 4096, batches, 4096, info) == 0
    del keep
    return {
        "valid": bool(info[0]),
        "total_layers": info[1],
        "total_spots": info[2],
        "max_spots_per_batch": info[3],
        "layer_spans": [_lib.struct_to_dict(spans[i]) for i in range(info[4])],
        "batches": [_lib.struct_to_dict(batches[i]) for i in range(info[5])],
    }


def _check(beam, m):
    got = operator_batch_plan(beam, m)
    want = oracle_plan(beam, m)
    assert got == want
    if REF_LIB.exists():
        assert got == _reference_plan(beam, m)
    return got


def test_seeded_beams_match_the_restatement():
    rng = np.random.Generator(np.random.PCG64(SEED))
    for _ in range(200):
        layers = int(rng.integers(1, 30))
        counts = rng.integers(0, 40, layers)
        counts[rng.random(layers) < 0.3] = 0
        m = int(rng.integers(-3, 120))
        plan = _check(_beam(counts), m)
        if counts.sum() > 0:
            assert plan["valid"]
            assert sum(b["spot_count"] for b in plan["batches"]) == counts.sum()
            assert all(b["first_layer_index"] >= 0 and counts[b["first_layer_index"]] > 0 for b in plan["batches"])


@pytest.mark.parametrize("case", [
    dict(counts=[]),                                   # no layers
    dict(counts=[3, 4], n_energies=3),                 # energies disagree with the layers
    dict(counts=[3, -1, 4]),                           # negative count
    dict(counts=[0, 0]),                               # no spots
    dict(counts=[3, 4], weights=6),                    # weights of the wrong size
    dict(counts=[3, 4], positions=15),                 # 15 // 2 == 7: accepted as the reference does
    dict(counts=[3, 4], positions=12),                 # 12 // 2 != 7
    dict(counts=[3, 4], directions=22),                # 22 // 3 == 7: accepted
    dict(counts=[3, 4], directions=20),                # 20 // 3 != 7
    dict(counts=[5, 0, 2], cutoffs=False),             # no cut-offs: 0 in every span
])
@pytest.mark.parametrize("m", [0, 1, 2, 7, 1000])
def test_edge_cases_match_the_restatement(case, m):
    case = dict(case)
    _check(_beam(case.pop("counts"), **case), m)


def test_headline_beam_plan(hetero_case):
    beam = hetero_case["beam"]
    plan = _check(beam, 256)
    assert plan["valid"] and plan["total_layers"] == len(beam["energies"])
    assert plan["total_spots"] == int(np.sum(beam["layer_spot_counts"]))
