"""torch.autograd binding of the solver's adjoint, for checking gradients.

:class:`EVPFunction` runs the subcycle loop forward through
``evp1d_run_checkpointed`` and its backward through ``evp1d_adjoint``, so
that torch's own tools (``torch.autograd.gradcheck``, losses built from torch
operations) can exercise the hand-written adjoint.  Tensors are CPU float64
([na] per-point fields); the solver keeps the state on the GPU.  The library
is the only compute path: nothing here differentiates the forward itself.
"""
from __future__ import annotations

import numpy as np
import torch

from . import EVP1D, FieldSet

INPUTS = ("strength", "Cw", "forcex", "forcey")


class EVPFunction(torch.autograd.Function):
    """(strength, Cw, forcex, forcey) -> (uvel, vvel) at the list points after
    ndte subcycles of ``problem`` on ``solver`` (an :class:`evp1d.EVP1D` built
    for it).  ``interval`` is the checkpoint interval of the recording (0:
    sized to device memory)."""

    @staticmethod
    def forward(ctx, solver: EVP1D, problem, ndte: int, interval: int,
                strength, Cw, forcex, forcey):
        pr = problem.copy()
        for name, t in zip(INPUTS, (strength, Cw, forcex, forcey)):
            pr.f[name] = t.detach().cpu().numpy().astype(np.float64).copy()
        fs = FieldSet.from_problem(pr)
        solver.run_checkpointed(int(ndte), fs, int(interval))
        ctx.solver, ctx.problem, ctx.ndte, ctx.interval = solver, pr, int(ndte), int(interval)
        ctx.recorded = solver.record_id = getattr(solver, "record_id", 0) + 1
        na = pr.na
        return (torch.from_numpy(fs.uvel[:na].copy()), torch.from_numpy(fs.vvel[:na].copy()))

    @staticmethod
    def backward(ctx, gu, gv):
        s = ctx.solver
        if getattr(s, "record_id", None) != ctx.recorded or not s.adjoint_info()["valid"]:
            # the solver recorded another forward since: record this one again
            s.run_checkpointed(ctx.ndte, FieldSet.from_problem(ctx.problem), ctx.interval)
            ctx.recorded = s.record_id = s.record_id + 1
        gu = np.zeros(s.na) if gu is None else gu.detach().cpu().numpy()
        gv = np.zeros(s.na) if gv is None else gv.detach().cpu().numpy()
        g = s.adjoint(gu, gv, want=INPUTS)
        return (None, None, None, None) + tuple(torch.from_numpy(g[k]) for k in INPUTS)


def evp_velocities(solver: EVP1D, problem, ndte: int, strength, Cw, forcex, forcey,
                   interval: int = 0):
    """Final list-point velocities as differentiable functions of the four
    fields (CPU float64 tensors of shape [na])."""
    return EVPFunction.apply(solver, problem, ndte, interval, strength, Cw, forcex, forcey)
