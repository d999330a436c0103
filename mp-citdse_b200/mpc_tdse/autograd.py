"""torch.autograd.Function over the adjoint entry points of libmpc_tdse.so.

``ControlObjective.apply(u, problem)`` returns J(u) -- the yield above the
context's threshold (or a target population) at the end of the fixed-step
propagation whose field is the pulse plus the piecewise-cubic perturbation
sampled by ``u`` -- as a 0-d float64 tensor.  ``backward`` multiplies the
adjoint gradient dJ/du (mpc_objective_backward) by the incoming gradient.
The forward pass keeps checkpoints in the context; the backward pass
recomputes between them.

``BatchControlObjective.apply(U, problem)`` does the same for B pulses at
once (U: [B, K], J: [B]) through mpc_batch_objective /
mpc_batch_objective_backward, whose forward and adjoint stages run as FP64
tensor-core GEMMs over the whole batch.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch


@dataclass
class ControlProblem:
    ctx: object            # mpc_tdse.Context
    pulse: object          # mpc_tdse.Pulse
    T: float               # control window [0, T]
    t0: float
    dt: float
    steps: int
    x0: np.ndarray         # start state (complex)
    target: int = -1       # -1: ionisation yield
    ckpt_every: int = 64


class ControlObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u, problem):
        uh = u.detach().to("cpu", torch.float64).numpy()
        J = problem.ctx.objective(problem.pulse, uh, problem.T, problem.t0, problem.dt,
                                  problem.steps, problem.x0, problem.target, problem.ckpt_every)
        ctx.problem = problem
        ctx.u_device = u.device
        return torch.tensor(J, dtype=torch.float64, device=u.device)

    @staticmethod
    def backward(ctx, grad_out):
        g, _ = ctx.problem.ctx.objective_backward()
        g = torch.from_numpy(g).to(ctx.u_device)
        return grad_out * g, None


def control_objective(u, problem):
    return ControlObjective.apply(u, problem)


@dataclass
class BatchControlProblem:
    ctx: object            # mpc_tdse.Context
    pulses: list           # B mpc_tdse.Pulse
    T: np.ndarray          # [B] control windows [0, T_b]
    t0: float
    dt: float
    steps: int
    x0: np.ndarray         # [B, size] start states (complex)
    target: int = -1       # -1: yield above the context's threshold
    ckpt_every: int = 0    # <= 0: sized to the free device memory


class BatchControlObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U, problem):
        Uh = U.detach().to("cpu", torch.float64).numpy()
        J = problem.ctx.batch_objective(problem.pulses, Uh, problem.T, problem.t0, problem.dt,
                                        problem.steps, problem.x0, problem.target,
                                        problem.ckpt_every)
        ctx.problem = problem
        ctx.u_device = U.device
        return torch.from_numpy(J).to(U.device)

    @staticmethod
    def backward(ctx, grad_out):
        G, _ = ctx.problem.ctx.batch_objective_backward()
        G = torch.from_numpy(G).to(ctx.u_device)
        return grad_out[:, None] * G, None


def batch_control_objective(U, problem):
    return BatchControlObjective.apply(U, problem)
