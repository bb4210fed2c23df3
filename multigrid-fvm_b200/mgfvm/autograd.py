"""torch.autograd interface of the engine's derivatives.

`objective(inlet_u, amuf, prsc, cfg, cycles)` returns J — the inlet-to-outlet
pressure drop plus the mean outlet scalar of the level-0 state after `cycles`
V-cycles (mgfvm_objective) — as a differentiable torch scalar.  The forward pass
runs one batched tangent context on the GPU (mgfvm_gradient: every inlet face, amuf
and prsc as cases of one batch), so the backward pass only scales the stored exact
derivatives by the incoming gradient.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import torch

from .inputs import CaseConfig
from .solver import gradient


class Objective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, inlet_u, amuf, prsc, cfg: CaseConfig, cycles: int, device: int):
        c = dataclasses.replace(cfg, amuf=float(amuf), prsc=float(prsc))
        prof = inlet_u.detach().to("cpu", torch.float64).numpy()
        j, g_in, g_amuf, g_prsc = gradient(c, prof, cycles, device)
        ctx.save_for_backward(torch.from_numpy(np.ascontiguousarray(g_in)).to(inlet_u.device, inlet_u.dtype),
                              torch.tensor(g_amuf, dtype=torch.float64, device=amuf.device),
                              torch.tensor(g_prsc, dtype=torch.float64, device=prsc.device))
        return torch.tensor(j, dtype=torch.float64, device=inlet_u.device)

    @staticmethod
    def backward(ctx, grad_j):
        g_in, g_amuf, g_prsc = ctx.saved_tensors
        return grad_j * g_in, grad_j * g_amuf, grad_j * g_prsc, None, None, None


def objective(inlet_u: torch.Tensor, amuf: torch.Tensor, prsc: torch.Tensor, cfg: CaseConfig, cycles: int,
              device: int = 0) -> torch.Tensor:
    """J(inlet_u, amuf, prsc) after `cycles` V-cycles of `cfg` (its own amuf and prsc
    are replaced by the arguments); inlet_u holds one value per level-0 inlet face
    (cfg.nfy values)."""
    if inlet_u.numel() != cfg.nfy:
        raise ValueError(f"inlet_u holds {inlet_u.numel()} values; the case has {cfg.nfy} inlet faces")
    return Objective.apply(inlet_u, amuf, prsc, cfg, int(cycles), int(device))
