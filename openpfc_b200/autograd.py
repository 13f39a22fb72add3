"""torch.autograd.Function over the hand-written adjoint (gradient harness only).

    psi_T = PfcEvolve.apply(psi0, r, model, n_steps, K)

runs the plain PFC step `n_steps` times on the GPU with snapshots every K
steps (opfc_forward_checkpointed) and, on backward, the adjoint through the
C ABI (opfc_adjoint).  psi0 and psi_T are CUDA tensors in the model's precision
with shape (N2, N1, N0); r is a 0-d tensor.  No torch kernel is involved in
either direction: torch only carries the buffers and the autograd graph.
"""
from __future__ import annotations

import torch

from . import FP64, PfcB200


class PfcEvolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, psi0: torch.Tensor, r: torch.Tensor, model: PfcB200, n_steps: int, K: int = 20):
        model.set_r(float(r))
        model.set_psi(psi0.detach().contiguous())
        model.forward_checkpointed(n_steps, K)
        out = torch.empty_like(psi0)
        model.get_psi(out)
        ctx.model = model
        ctx.r_dtype = r.dtype
        ctx.r_device = r.device
        return out

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        g0, gr, _ = ctx.model.adjoint(grad_out.detach().contiguous())
        return g0, torch.tensor(gr, dtype=ctx.r_dtype, device=ctx.r_device), None, None, None


def make_model(n, dx, precision=FP64, dt=0.5, r=-0.25, device=0) -> PfcB200:
    m = PfcB200(n, dx, r=r, precision=precision, device=device)
    m.initialize(dt)
    return m
