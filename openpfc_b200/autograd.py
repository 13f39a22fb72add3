"""torch.autograd.Function over the hand-written adjoint (gradient harness only).

    psi_T = PfcEvolve.apply(psi0, r, model, n_steps, K)

runs the model's step `n_steps` times on the GPU with snapshots every K steps
(opfc_forward_checkpointed) and, on backward, the adjoint through the C ABI
(opfc_adjoint).  The model is any of the package's models with an adjoint
(plain, filtered, Tungsten, Aluminum without a moving gradient); psi0 and psi_T
are CUDA tensors in the model's precision with shape (N2, N1, N0); r is a 0-d
tensor for the models with r (plain, filtered) and None otherwise.  No torch
kernel is involved in either direction: torch only carries the buffers and the
autograd graph.
"""
from __future__ import annotations

import torch

from . import FP64, PfcB200


class PfcEvolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, psi0: torch.Tensor, r, model, n_steps: int, K: int = 20):
        if r is not None:
            model.set_r(float(r))
        model.set_psi(psi0.detach().contiguous())
        model.forward_checkpointed(n_steps, K)
        out = torch.empty_like(psi0)
        model.get_psi(out)
        ctx.model = model
        ctx.has_r = r is not None
        ctx.r_dtype = r.dtype if r is not None else None
        ctx.r_device = r.device if r is not None else None
        return out

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        g0, gr, _ = ctx.model.adjoint(grad_out.detach().contiguous())
        g_r = torch.tensor(gr, dtype=ctx.r_dtype, device=ctx.r_device) if ctx.has_r else None
        return g0, g_r, None, None, None


def make_model(n, dx, precision=FP64, dt=0.5, r=-0.25, device=0) -> PfcB200:
    m = PfcB200(n, dx, r=r, precision=precision, device=device)
    m.initialize(dt)
    return m
