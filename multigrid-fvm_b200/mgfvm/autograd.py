"""torch.autograd interface of the engine's derivatives.

`objective(inlet_u, amuf, prsc, cfg, cycles)` returns J — the inlet-to-outlet
pressure drop plus the mean outlet scalar of the level-0 state after `cycles`
V-cycles (mgfvm_objective) — as a differentiable torch scalar.  The forward pass
runs one batched tangent context on the GPU (mgfvm_gradient: every inlet face, amuf
and prsc as cases of one batch), so the backward pass only scales the stored exact
derivatives by the incoming gradient.

`objective_batch(inlet_u, amuf, prsc, cfgs, cycles)` does the same for a batch of B
cases at once (inlet_u: (B, nfy), amuf and prsc: (B,)) in one context, by reverse
mode (mgfvm_adjoint): one adjoint run gives every case's whole gradient.
"""
from __future__ import annotations

import dataclasses
from typing import Sequence

import numpy as np
import torch

from .inputs import CaseConfig
from .solver import Solver, gradient


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


class ObjectiveBatch(torch.autograd.Function):
    @staticmethod
    def forward(ctx, inlet_u, amuf, prsc, cfgs, cycles: int, device: int):
        prof = inlet_u.detach().to("cpu", torch.float64).numpy()
        a = amuf.detach().to("cpu", torch.float64).numpy()
        p = prsc.detach().to("cpu", torch.float64).numpy()
        cases = [dataclasses.replace(c, amuf=float(a[k]), prsc=float(p[k])) for k, c in enumerate(cfgs)]
        with Solver(cases, device=device) as s:
            for k in range(len(cases)):
                s.set_inlet_profile(k, prof[k])
            s.adjoint(cycles)
            res = [s.adjoint_gradient(k) for k in range(len(cases))]
        j = torch.tensor([r[0] for r in res], dtype=torch.float64, device=inlet_u.device)
        g_in = torch.from_numpy(np.stack([r[1] for r in res])).to(inlet_u.device, inlet_u.dtype)
        g_a = torch.tensor([r[2] for r in res], dtype=torch.float64, device=amuf.device)
        g_p = torch.tensor([r[3] for r in res], dtype=torch.float64, device=prsc.device)
        ctx.save_for_backward(g_in, g_a, g_p)
        return j

    @staticmethod
    def backward(ctx, grad_j):
        g_in, g_a, g_p = ctx.saved_tensors
        return grad_j[:, None] * g_in, grad_j * g_a, grad_j * g_p, None, None, None


def objective_batch(inlet_u: torch.Tensor, amuf: torch.Tensor, prsc: torch.Tensor, cfgs: Sequence[CaseConfig],
                    cycles: int, device: int = 0) -> torch.Tensor:
    """J of each of B cases after `cycles` V-cycles (shape (B,)): inlet_u (B, nfy) holds
    every case's per-face inlet profile, amuf and prsc (B,) replace each case's own.
    The cases must share nfy, the smoother and its sweep counts; sizes, obstacles and
    physics may differ.  The gradient comes from one reverse-mode run of the batch."""
    cfgs = list(cfgs)
    b = len(cfgs)
    if b == 0:
        raise ValueError("no cases")
    nfy = cfgs[0].nfy
    if any(c.nfy != nfy for c in cfgs):
        raise ValueError("the cases of a batch must share nfy (one inlet profile row each)")
    if tuple(inlet_u.shape) != (b, nfy):
        raise ValueError(f"inlet_u has shape {tuple(inlet_u.shape)}; expected ({b}, {nfy})")
    if tuple(amuf.shape) != (b,) or tuple(prsc.shape) != (b,):
        raise ValueError(f"amuf and prsc must have shape ({b},)")
    return ObjectiveBatch.apply(inlet_u, amuf, prsc, cfgs, int(cycles), int(device))
