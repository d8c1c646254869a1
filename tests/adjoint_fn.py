"""Test-only torch.autograd.Function over fx_forward_record / fx_backward.

It exists to check the hand-written adjoint against central finite
differences; the library's own forward/backward API is the C one.
theta = (alpha, beta, gamma, g11, g44, v_amp) as a float64 tensor.
"""
import numpy as np
import torch

from ferrox_b200 import api


class HysteresisLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, make, target, v_shape, checkpoint_every):
        fx = make()
        for name, v in zip(api.GRADS[:5], theta[:5].tolist()):
            fx.set_param(name, v)
        loss = fx.forward_record(target, float(theta[5]), v_shape, checkpoint_every)
        ctx.fx = fx
        return theta.new_tensor(loss)

    @staticmethod
    def backward(ctx, gout):
        g = ctx.fx.backward()
        ctx.fx.close()
        return gout * torch.from_numpy(np.asarray(g)).to(gout.dtype), None, None, None, None


def loss_and_grad(theta, make, target, v_shape, k):
    t = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    L = HysteresisLoss.apply(t, make, target, v_shape, k)
    L.backward()
    return float(L.detach()), t.grad.numpy().copy()


def loss_with(theta, q, dx, make, target, v_shape, k):
    """The loss with theta[q] moved by dx (no gradient kept)."""
    t = np.array(theta, dtype=np.float64)
    t[q] += dx
    with torch.no_grad():
        return float(HysteresisLoss.apply(torch.tensor(t), make, target, v_shape, k))
