"""Operator mode: the spot-preserving batch plan of a beam
(`buildRTDOperatorBatchPlan`, include/core/rtd_operator_mode.h:43-111) through
`pbs_operator_batch_plan`, and the dose-influence export in compressed sparse
columns (`DoseEngine.influence_csc`, `pbs_context_influence_csc`)."""
from __future__ import annotations

import ctypes as C

from . import _lib


def operator_batch_plan(beam: dict, max_spots_per_batch: int) -> dict:
    """The beam's layer spans and spot batches, as the reference's
    RTDOperatorBatchPlan (rtd_operator_mode.h:34-41): keys valid, total_layers,
    total_spots, max_spots_per_batch, layer_spans and batches (lists of dicts)."""
    lib = _lib.load()
    bd, keep = _lib.beam_desc(beam)
    info = (C.c_int * 6)()
    _lib.check(lib.pbs_operator_batch_plan(C.byref(bd), int(max_spots_per_batch), None, 0, None, 0, info))
    spans = (_lib.PbsOperatorLayerSpan * max(info[4], 1))()
    batches = (_lib.PbsOperatorBatch * max(info[5], 1))()
    _lib.check(lib.pbs_operator_batch_plan(C.byref(bd), int(max_spots_per_batch), spans, info[4], batches, info[5],
                                           info))
    del keep
    return {
        "valid": bool(info[0]),
        "total_layers": info[1],
        "total_spots": info[2],
        "max_spots_per_batch": info[3],
        "layer_spans": [_lib.struct_to_dict(spans[i]) for i in range(info[4])],
        "batches": [_lib.struct_to_dict(batches[i]) for i in range(info[5])],
    }
