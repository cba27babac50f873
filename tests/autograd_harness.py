"""torch.autograd.Function around the library's adjoint force: a thin ctypes
test harness, not part of the product (the product boundary is the C ABI).

    logdet = LogDet.apply(x, ctx, mode)

Forward is one ephmc_eval (log det of M_hat = 1 + B_0...B_{Nt-1}); backward
is the force the same call computed, p_dot = flavors * d log det / dx
(simulation/organic_hmc.c:86-134), scaled by the incoming gradient."""
import torch


class LogDet(torch.autograd.Function):
    @staticmethod
    def forward(fctx, x, ctx, mode="adjoint"):
        x = x.detach().contiguous()
        p_dot = torch.empty_like(x)
        ld, _ = ctx.eval(x, p_dot, mode=mode)
        fctx.save_for_backward(p_dot)
        fctx.flavors = ctx.flavors
        return x.new_tensor(ld)

    @staticmethod
    def backward(fctx, grad):
        (p_dot,) = fctx.saved_tensors
        return grad * p_dot / fctx.flavors, None, None
