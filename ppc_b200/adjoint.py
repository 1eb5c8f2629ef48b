"""Poisson log-likelihood of per-DOM charges as a differentiable function of the ice model.

    params = torch.tensor(np.stack([be, ba]), dtype=torch.float64, requires_grad=True)
    ll = IceLikelihood.apply(params, ppc, bunches, observed, scale, events)
    ll.backward()          # params.grad: d LL / d (be_j, ba_j), file order

The forward pass sets the coefficients (ppcb_set_ice), propagates the bunches once while
recording the provenance of every hit, and the same call replays the detected photons to
form the gradient (ppcb_gradient); backward returns that gradient.  The per-layer sums are
accumulated in FP64 on the GPU.  `observed` holds per-DOM charges (events = 0) or per
(event, DOM) charges, shape (events, gsize), the event being each bunch's q.
"""
import numpy as np
import torch


class IceLikelihood(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, ppc, bunches, observed, scale=1.0, events=0):
        p = params.detach().cpu().numpy()
        ppc.set_ice(p[0].astype(np.float32), p[1].astype(np.float32))
        r = ppc.gradient(bunches, observed=observed, scale=scale, events=events)
        g = torch.from_numpy(np.stack([r["g_be"], r["g_ba"]])).to(params.dtype)
        ctx.save_for_backward(g)
        ctx.info = r["info"]
        return torch.tensor(r["ll"], dtype=params.dtype)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None, None, None, None, None
