"""Beam-sharded dose over several GPUs, one process per GPU.

Beams are independent and a plan's dose is the sum of its beams' doses
(raytracedicom_wrapper.cu:2446-5661 loops over beams into one grid), so the
beams are divided among the ranks, every rank computes its beams into its own
FP64 dose grid, and a single reduction sums the grids on the destination rank.
No other data crosses ranks: this is the only collective of the path.

A single beam shards by energy layer in the same way: the layers of a beam are
independent once the beam is traced (raytracedicom_wrapper.cu:3917-5625 loops
over them into one grid), so each rank traces the whole beam (the cheap part),
computes only its share of the layers (the other layers' spots at zero weight,
which leaves their rays dead and their tiles out of the superposition) and the
same single reduction sums the shares.

The functions take any engine with `reset_dose()`, `add_beam(beam)` and
`read_dose64(out)` (`cudaCalDoseRTD.DoseEngine` on a GPU) and any
`torch.distributed` process group (NCCL between GPUs; gloo works for CPU
tensors)."""
from __future__ import annotations

from typing import Sequence

import numpy as np


def beam_cost(beam) -> float:
    """Relative cost of a beam: spots x layers (the IDD and superposition work
    grows with both), from a beam dict; 1.0 when the beam carries no spot list."""
    if isinstance(beam, dict):
        layers = max(len(np.asarray(beam.get("energies", [1])).reshape(-1)), 1)
        counts = beam.get("layer_spot_counts")
        if counts is not None:
            return float(np.sum(counts)) * layers
        sub = beam.get("subspot_data")
        if sub is not None:
            return float(np.asarray(sub).shape[1]) * layers
        return float(layers)
    return 1.0


def assign_beams(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time assignment of beams to `world` ranks: beams sorted
    by descending cost (ties by index) go to the least loaded rank (ties by rank).
    Deterministic, so every rank computes the same assignment without talking."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(costs[i])
    for lst in out:
        lst.sort()
    return out


def assign_layers(beam: dict, world: int) -> list[list[int]]:
    """Layers of `beam` per rank: longest-processing-time on the layers' spot counts
    (every layer costs at least 1), deterministic as assign_beams."""
    counts = np.asarray(beam["layer_spot_counts"]).reshape(-1)
    return assign_beams([max(float(c), 1.0) for c in counts], world)


def layer_share(beam: dict, layers: Sequence[int]) -> dict:
    """The beam with only `layers` carrying spot weight. Spot positions, energies and
    everything the plan is made from stay, so every share has the whole beam's ray
    grid, lattice and cut-off steps, and the shares' doses add up to the beam's."""
    counts = np.asarray(beam["layer_spot_counts"]).astype(np.int64).reshape(-1)
    keep = np.zeros(int(counts.sum()), bool)
    starts = np.concatenate([[0], np.cumsum(counts)])
    for l in layers:
        keep[starts[l]:starts[l + 1]] = True
    out = dict(beam)
    out["spot_weights"] = np.where(keep, np.asarray(beam["spot_weights"], np.float32), np.float32(0.0))
    return out


def beam_layers_dose(engine, beam: dict, dose64, rank: int, world: int, dst: int = 0, group=None):
    """This rank's share of one beam's layers, reduced on `dst`. A rank without
    layers (more ranks than layers) adds nothing and still joins the reduction.
    Returns (tensor, assigned layer indices)."""
    mine = assign_layers(beam, world)[rank]
    engine.reset_dose()
    if mine:
        engine.add_beam(layer_share(beam, mine))
    engine.read_dose64(dose64)
    if world > 1:
        reduce_dose(dose64, dst=dst, group=group)
    return dose64, mine


def reduce_dose(dose64, dst: int = 0, group=None):
    """Sum the ranks' FP64 dose grids on `dst` (in place); returns the tensor."""
    import torch.distributed as dist

    dist.reduce(dose64, dst=dst, op=dist.ReduceOp.SUM, group=group)
    return dose64


def plan_dose(engine, beams: Sequence, dose64, rank: int, world: int, dst: int = 0, group=None,
              nuclear_correction: bool = False):
    """This rank's share of a multi-beam plan, reduced on `dst`.

    Resets the engine's dose grid, adds the beams assigned to `rank`, reads the
    FP64 grid into `dose64` (a torch tensor on the collective's device) and
    reduces it. On `dst` the returned tensor holds the dose of the whole plan;
    other ranks return their partial grid. Returns (tensor, assigned beam indices)."""
    mine = assign_beams([beam_cost(b) for b in beams], world)[rank]
    engine.reset_dose()
    for i in mine:
        if nuclear_correction:
            engine.add_beam(beams[i], nuclear_correction=True)
        else:
            engine.add_beam(beams[i])
    engine.read_dose64(dose64)
    if world > 1:
        reduce_dose(dose64, dst=dst, group=group)
    return dose64, mine
