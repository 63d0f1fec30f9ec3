"""CPU restatement of the reference's operator-mode batch plan (test
infrastructure only: the checker of `pbs_operator_batch_plan`, never a product
path). Follows buildRTDOperatorBatchPlan, include/core/rtd_operator_mode.h:43-111:
validation order and early returns (lines 45-68), layer spans in layer order
(72-84), batches of max(1, maxSpotsPerBatch) consecutive spots (86-108) whose
first/last layer is the first non-empty span holding the spot (87-98)."""
from __future__ import annotations

import numpy as np


def operator_batch_plan(beam: dict, max_spots_per_batch: int) -> dict:
    def n(key):
        v = beam.get(key)
        return 0 if v is None else int(np.asarray(v).size)

    counts = [int(c) for c in np.asarray(beam.get("layer_spot_counts", []), dtype=np.int64).ravel()]
    energies = np.asarray(beam.get("energies", []), dtype=np.float32).ravel()
    cutoffs = np.asarray(beam.get("layer_longitudinal_cutoffs", []), dtype=np.float32).ravel()
    plan = {"valid": False, "total_layers": len(counts), "total_spots": 0, "max_spots_per_batch": 0,
            "layer_spans": [], "batches": []}
    if plan["total_layers"] <= 0 or energies.size != plan["total_layers"]:
        return plan
    if any(c < 0 for c in counts):
        return plan
    total = sum(counts)
    plan["total_spots"] = total
    if total <= 0:
        return plan
    if n("spot_weights") and n("spot_weights") != total:
        return plan
    if n("spot_positions") and n("spot_positions") // 2 != total:
        return plan
    if n("spot_beam_directions") and n("spot_beam_directions") // 3 != total:
        return plan
    running = 0
    for layer, c in enumerate(counts):
        plan["layer_spans"].append({"layer_index": layer, "spot_begin": running, "spot_count": c,
                                    "energy": float(energies[layer]),
                                    "longitudinal_cutoff": float(cutoffs[layer]) if layer < cutoffs.size else 0.0})
        running += c
    m = max(1, int(max_spots_per_batch))
    plan["max_spots_per_batch"] = m

    def layer_of(spot):
        for s in plan["layer_spans"]:
            if s["spot_count"] > 0 and s["spot_begin"] <= spot < s["spot_begin"] + s["spot_count"]:
                return s["layer_index"]
        return -1

    for index, begin in enumerate(range(0, total, m)):
        cnt = min(m, total - begin)
        plan["batches"].append({"batch_index": index, "spot_begin": begin, "spot_count": cnt,
                                "first_layer_index": layer_of(begin), "last_layer_index": layer_of(begin + cnt - 1)})
    plan["valid"] = bool(plan["layer_spans"]) and bool(plan["batches"])
    return plan
