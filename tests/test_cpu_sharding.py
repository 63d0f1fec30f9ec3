"""Beam sharding and the dose reduction with two gloo ranks on the CPU; the
per-rank dose comes from the oracle standing in for a GPU engine."""
import os
import socket

import numpy as np
import pytest

from subsecondpbs_b200 import sharding


def test_assignment_is_balanced_and_complete():
    costs = [5.0, 1.0, 3.0, 3.0, 2.0, 8.0]
    for world in (1, 2, 3, 4, 8):
        parts = sharding.assign_beams(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
    assert sharding.assign_beams(costs, 2) == sharding.assign_beams(list(costs), 2)
    assert sharding.assign_beams([1.0, 1.0, 1.0], 2) == [[0, 2], [1]]


def test_beam_cost_counts_spots_and_layers(hetero_small_case):
    b = hetero_small_case["beam"]
    layers = len(b["energies"])
    assert sharding.beam_cost(b) == float(np.sum(b["layer_spot_counts"])) * layers


class OracleEngine:
    """CPU stand-in for DoseEngine with the oracle as the per-beam dose."""

    def __init__(self, case):
        self.case = case
        self.acc = None

    def reset_dose(self):
        self.acc = np.zeros_like(self.case["ct"], dtype=np.float64)

    def add_beam(self, beam):
        from oracle import oracle as O

        self.acc += O.dose(self.case, beams=[beam], threads=2)["dose"]

    def read_dose64(self, out):
        import torch

        out.copy_(torch.from_numpy(self.acc))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, result_path, fail_rank, mode="beams"):
    import sys
    from datetime import timedelta
    from pathlib import Path

    root = Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "tests"))
    import torch
    import torch.distributed as dist

    from subsecondpbs_b200 import phantoms

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=20))
    case = phantoms.heterogeneous_case(dims=(48, 48, 32), n_layers=2, target_radius_mm=10.0)
    beams = [phantoms.rotate_beam(case["beam"], a) for a in (0.0, 90.0, 180.0)]
    dose = torch.zeros(case["ct"].shape, dtype=torch.float64)
    status = "ok"
    try:
        if rank == fail_rank:
            raise RuntimeError("rank failed before its collective")
        if mode == "layers":
            out, mine = sharding.beam_layers_dose(OracleEngine(case), beams[1], dose, rank, world)
        else:
            out, mine = sharding.plan_dose(OracleEngine(case), beams, dose, rank, world)
        if rank == 0:
            np.save(result_path, out.numpy())
    except Exception as e:  # recorded for the parent; a peer's failure must surface as an error here
        status = f"error: {type(e).__name__}"
    Path(f"{result_path}.rank{rank}").write_text(status)
    if status == "ok":
        dist.destroy_process_group()


def _spawn(tmp_path, fail_rank, mode="beams"):
    import torch.multiprocessing as mp

    result = str(tmp_path / "dose.npy")
    mp.start_processes(_worker, args=(2, _free_port(), result, fail_rank, mode), nprocs=2, join=True,
                       start_method="spawn")
    return result


def test_two_ranks_sum_to_the_whole_plan(tmp_path):
    from oracle import oracle as O
    from subsecondpbs_b200 import phantoms

    result = _spawn(tmp_path, fail_rank=-1)
    case = phantoms.heterogeneous_case(dims=(48, 48, 32), n_layers=2, target_radius_mm=10.0)
    beams = [phantoms.rotate_beam(case["beam"], a) for a in (0.0, 90.0, 180.0)]
    whole = O.dose(case, beams=beams, threads=2)["dose"]
    got = np.load(result)
    assert np.abs(got - whole).max() <= 1e-12 * whole.max()
    assert (tmp_path / "dose.npy.rank1").read_text() == "ok"


def test_a_failed_rank_surfaces_as_an_error(tmp_path):
    _spawn(tmp_path, fail_rank=1)
    assert (tmp_path / "dose.npy.rank1").read_text().startswith("error")
    assert (tmp_path / "dose.npy.rank0").read_text().startswith("error")


def test_layer_assignment_covers_every_layer_once(hetero_small_case):
    beam = hetero_small_case["beam"]
    L = len(beam["energies"])
    for world in (1, 2, 3, 5):
        parts = sharding.assign_layers(beam, world)
        assert sorted(l for p in parts for l in p) == list(range(L))


def test_layer_shares_sum_to_the_beam():
    """The shares' doses add up to the whole beam's: layers are independent once the
    beam is traced, and a layer without weight deposits nothing."""
    from oracle import oracle as O
    from subsecondpbs_b200 import phantoms

    case = phantoms.heterogeneous_case(dims=(48, 48, 32), n_layers=3, target_radius_mm=10.0)
    beam = case["beam"]
    whole = O.dose(case, threads=2)["dose"]
    parts = [O.dose(case, beams=[sharding.layer_share(beam, [l])], threads=2)["dose"] for l in range(3)]
    assert np.abs(sum(parts) - whole).max() <= 1e-12 * whole.max()
    assert all(p.max() > 0 for p in parts)


def test_two_ranks_shard_one_beam_by_layer(tmp_path):
    from oracle import oracle as O
    from subsecondpbs_b200 import phantoms

    result = _spawn(tmp_path, fail_rank=-1, mode="layers")
    case = phantoms.heterogeneous_case(dims=(48, 48, 32), n_layers=2, target_radius_mm=10.0)
    beam = phantoms.rotate_beam(case["beam"], 90.0)
    whole = O.dose(case, beams=[beam], threads=2)["dose"]
    got = np.load(result)
    assert np.abs(got - whole).max() <= 1e-12 * whole.max()
    assert (tmp_path / "dose.npy.rank1").read_text() == "ok"
