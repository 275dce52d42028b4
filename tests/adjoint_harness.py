"""torch.autograd.Function over the differentiated-window C ABI.

Test harness only: the solver itself stays C++; this wrapper lets the tests
drive the window through torch's autograd (J.backward()) and compare with
finite differences.  Forward: pfem2gpu_window_forward_device; backward:
pfem2gpu_window_backward_device.  Inputs: v0 (n, dim), V and Vold
(dim, n_dofs), float64 CUDA tensors.
"""
import torch


class ParticleWindow(torch.autograd.Function):
    @staticmethod
    def forward(ctx, v0, V, Vold, handler, steps, checkpoint_every):
        torch.cuda.synchronize()  # inputs are written on torch's stream, the window runs on the handler's
        U = torch.empty_like(V)
        handler.window_forward_device(steps, checkpoint_every, V.detach().contiguous(),
                                      None if Vold is None else Vold.detach().contiguous(),
                                      v0.detach().contiguous(), U)
        handler.synchronize()
        ctx.handler = handler
        ctx.shapes = (v0.shape, V.shape, Vold is not None)
        return U

    @staticmethod
    def backward(ctx, gU):
        vshape, Vshape, has_old = ctx.shapes
        g_v0 = torch.empty(vshape, dtype=torch.float64, device=gU.device)
        g_V = torch.empty(Vshape, dtype=torch.float64, device=gU.device)
        g_Vold = torch.empty(Vshape, dtype=torch.float64, device=gU.device) if has_old else None
        torch.cuda.synchronize()
        ctx.handler.window_backward_device(gU.contiguous().to(torch.float64), g_v0, g_V, g_Vold)
        return g_v0, g_V, g_Vold, None, None, None


def window(handler, v0, V, Vold=None, steps=1, checkpoint_every=1):
    return ParticleWindow.apply(v0, V, Vold, handler, steps, checkpoint_every)
