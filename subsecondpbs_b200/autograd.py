"""The dose of a plan as a differentiable function of its spot weights.

`SpotWeightDose.apply(weights, engine, beams)` returns the FP64 dose grid
([Z][Y][X], CUDA) of `beams` computed by `engine` (a `DoseEngine` holding the
tables, CT and dose grid) with the spot weights taken from `weights`, a 1-D
tensor of every beam's weights concatenated in beam order. Its backward pass runs
the library's hand-written adjoint (pbs_context_adjoint_beam): the transposes of
the transfer, the tile superposition and the spot -> ray convolution, one beam at a
time, at the forward's tile radii and live rays. Everything after the dose (the
objective, its reduction) is ordinary torch code, in FP64 on the GPU.
"""
from __future__ import annotations

import numpy as np
import torch


def spot_counts(beams) -> list[int]:
    return [int(np.sum(b["layer_spot_counts"])) for b in beams]


def with_weights(beam: dict, w: np.ndarray) -> dict:
    out = dict(beam)
    out["spot_weights"] = np.ascontiguousarray(w, dtype=np.float32)
    return out


class SpotWeightDose(torch.autograd.Function):
    @staticmethod
    def forward(ctx, weights, engine, beams):
        w = weights.detach().to(torch.float32).cpu().numpy()
        sizes = spot_counts(beams)
        if sum(sizes) != w.size:
            raise ValueError(f"{w.size} weights for {sum(sizes)} spots")
        prepared, off = [], 0
        for b, n in zip(beams, sizes):
            prepared.append(engine.prepare_beam(with_weights(b, w[off:off + n])))
            off += n
        engine.reset_dose()
        for p in prepared:
            engine.add_beam(p)
        dims = engine.dose_dims
        dose = torch.empty((dims[2], dims[1], dims[0]), dtype=torch.float64, device=f"cuda:{engine.gpu_id}")
        engine.read_dose64(dose)
        engine.synchronize()
        ctx.engine, ctx.prepared, ctx.sizes = engine, prepared, sizes
        ctx.weight_dtype, ctx.weight_device = weights.dtype, weights.device
        return dose

    @staticmethod
    def backward(ctx, grad):
        g = grad.detach().to(torch.float64).contiguous()
        torch.cuda.synchronize(g.device)
        parts = [ctx.engine.adjoint_beam(p, g, n) for p, n in zip(ctx.prepared, ctx.sizes)]
        gw = torch.from_numpy(np.concatenate(parts)).to(device=ctx.weight_device, dtype=ctx.weight_dtype)
        return gw, None, None


def plan_dose(weights, engine, beams):
    """Differentiable dose of `beams` at `weights` (see SpotWeightDose)."""
    return SpotWeightDose.apply(weights, engine, beams)
