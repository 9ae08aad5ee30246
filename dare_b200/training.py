"""On-GPU training of the learned linear preconditioner.

The training distribution is the one the learned solver is meant for:
periodic TVD (van Leer) convection-diffusion operators on one grid, half of
them with constant D = 1e-4 and half with the log-normal, box-filtered D
(mu = ln 1e-4, sigma = 1, 5-cell filter), a random divergence-free
streamfunction velocity at a cell Peclet number drawn from [1, 10], and dt at
CFL 0.5.  Each operator is stepped in time; every implicit step is solved by
the plain FP64 Jacobi-BiCGStab2, whose iterates become (residual, error)
pairs for the network (``dare_unet_train_on_system``), followed by Adam steps
on minibatches drawn from the pair ring -- forward and backward passes run in
the library's tcgen05 convolution kernels.
"""
from __future__ import annotations

import numpy as np

from . import Assembly, Context, DeviceArray, Field, Grid, LearnedPreconditioner, MatrixSystem, face_average
from . import workloads as W


def sample_case(n: int, seed: int, device: str) -> dict:
    """One operator of the training distribution (synthetic, seeded)."""
    rng = np.random.default_rng(seed)
    peclet = float(rng.uniform(1.0, 10.0))
    if rng.integers(0, 2):
        case = W.heterogeneous(n=n, seed=seed, peclet=peclet, device=device)
    else:
        case = W.tvd_convection_diffusion(n=n, seed=seed, peclet=peclet, device=device)
    case["peclet"] = peclet
    return case


class Operator:
    """A grid, a two-level field and an assembled system for one sampled case."""

    def __init__(self, ctx: Context, case: dict):
        import torch
        self.case = case
        self.grid = Grid(ctx, case["n"], case["size"], 2, case["periodic"])
        self.field = Field(self.grid, 2)
        phi0 = case["phi0"].reshape(-1)
        phi0 = phi0.cpu().numpy() if hasattr(phi0, "cpu") else np.asarray(phi0)
        self.phi0 = np.ascontiguousarray(phi0, dtype=np.float64)
        self.reset()
        dev = case["face_vel"][0].device if hasattr(case["face_vel"][0], "device") else "cuda:0"
        self.vel = [DeviceArray.from_tensor(torch.as_tensor(case["face_vel"][d], device=dev)) for d in range(3)]
        if "cell_D" in case:
            cell_D = torch.as_tensor(case["cell_D"], device=dev).contiguous()
            self.faceD = [DeviceArray.from_tensor(torch.empty(self.grid.face_shape(d), dtype=torch.float64,
                                                              device=dev)) for d in range(3)]
            face_average(self.grid, cell_D.data_ptr(), self.faceD)
            self.asm = Assembly(dt=case["dt"], face_D=tuple(self.faceD), face_vel=tuple(self.vel))
        else:
            self.asm = Assembly(dt=case["dt"], D=case["D"], face_vel=tuple(self.vel))
        self.system = MatrixSystem(self.grid)

    def reset(self):
        self.field.upload(self.phi0, 0)
        self.field.upload(self.phi0, 1)

    def assemble(self):
        self.system.build(self.field, self.asm)

    def advance(self):
        """Accept the system's solution as the new time level."""
        self.system.copy_to(self.field)
        self.field.exchange_halo()
        self.field.copy_to_old()


def train(net: LearnedPreconditioner, ctx: Context, n: int, operators: int = 16, steps_per_operator: int = 4,
          params=None, tol: float = 1e-10, seed: int = 0, device: str = "cuda:0", log=None) -> list[dict]:
    """Train `net` on `operators` sampled operators, `steps_per_operator` implicit
    steps each.  Returns one report per step (pairs added, losses)."""
    reports = []
    for o in range(operators):
        op = Operator(ctx, sample_case(n, seed + 7919 * o, device))
        for s in range(steps_per_operator):
            op.assemble()
            rep = net.train_on_system(op.system, tol, params)
            rep["operator"] = o
            rep["peclet"] = op.case["peclet"]
            reports.append(rep)
            if log:
                log(rep)
            op.advance()
    return reports
