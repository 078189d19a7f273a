"""Optional PyTorch binding: GSE-k energy and forces as a differentiable op.

    E, F = gse_energy_forces(xyz, q, ctx)

xyz (n, 3) and q (n,) are CUDA tensors; ctx is a gse_b200.gse.Context.  E is a
0-d float64 tensor, F an (n, 3) float64 tensor.  Backward calls the
library's hand-written adjoint (gse_adjoint), which recomputes the grids
from the inputs instead of keeping them between forward and backward.
Everything runs on the current torch stream.
"""
from __future__ import annotations

import torch

from .gse import Context


class GSEEnergyForces(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xyz, q, gse_ctx: Context):
        n = xyz.shape[0]
        dtype = torch.float64 if gse_ctx.precision == "fp64" else torch.float32
        xyzq = torch.cat([xyz.detach(), q.detach()[:, None]], dim=1).to(dtype).contiguous()
        gse_ctx.set_stream(torch.cuda.current_stream(xyz.device).cuda_stream)
        F = torch.empty(3, n, dtype=torch.float64, device=xyz.device)
        E = torch.empty(1, dtype=torch.float64, device=xyz.device)
        gse_ctx.forward(n, xyzq, F[0], F[1], F[2], energy_out=E)
        ctx.gse = gse_ctx
        ctx.save_for_backward(xyzq)
        ctx.in_dtypes = (xyz.dtype, q.dtype)
        return E[0], F.t()

    @staticmethod
    def backward(ctx, gE, gF):
        (xyzq,) = ctx.saved_tensors
        n = xyzq.shape[0]
        gse_ctx = ctx.gse
        gse_ctx.set_stream(torch.cuda.current_stream(xyzq.device).cuda_stream)
        out = torch.empty(4, n, dtype=torch.float64, device=xyzq.device)
        dLdE = float(gE.item()) if gE is not None else 0.0
        if gF is not None:
            g = gF.t().to(torch.float64).contiguous()
            gse_ctx.adjoint(n, xyzq, dLdE, g[0], g[1], g[2], out[0], out[1], out[2], out[3])
        else:
            gse_ctx.adjoint(n, xyzq, dLdE, None, None, None, out[0], out[1], out[2], out[3])
        dq = out[0].to(ctx.in_dtypes[1])
        dxyz = out[1:].t().to(ctx.in_dtypes[0])
        return dxyz, dq, None


def gse_energy_forces(xyz: torch.Tensor, q: torch.Tensor, ctx: Context):
    return GSEEnergyForces.apply(xyz, q, ctx)
