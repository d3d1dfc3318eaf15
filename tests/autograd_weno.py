"""TEST-ONLY torch.autograd wrapper of one WENO sweep over the C ABI.

forward: (vL, vR) = sweep(v_rs_ws) through weno_sb_weno_dev;
backward: gv = VJP through weno_sb_vjp_dev (beta and the weights are
recomputed from v, nothing is saved but v itself)."""
import torch

from wenostandalone_b200 import api


class WenoSweep(torch.autograd.Function):
    @staticmethod
    def forward(ctx, v, grid, d, order, coefs, flags):
        n = 1
        for s in grid.face_shape(d):
            n *= s
        vL = torch.zeros(n, dtype=torch.float64, device=v.device)
        vR = torch.zeros(n, dtype=torch.float64, device=v.device)
        api.weno(grid, d, order, v.detach(), coefs, vL, vR, flags=flags)
        ctx.save_for_backward(v)
        ctx.args = (grid, d, order, coefs, flags)
        return vL, vR

    @staticmethod
    def backward(ctx, gL, gR):
        (v,) = ctx.saved_tensors
        grid, d, order, coefs, flags = ctx.args
        gv = torch.empty_like(v)
        api.vjp(grid, d, order, v.detach(), coefs, gL.contiguous(), gR.contiguous(), gv, flags=flags)
        return gv, None, None, None, None, None
