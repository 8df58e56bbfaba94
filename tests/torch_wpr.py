"""Test-side torch binding of the weighted-PageRank adjoint: a
torch.autograd.Function whose forward and backward call the C ABI
(gg_pagerank_weighted_fwd / gg_pagerank_weighted_bwd) on CPU tensors."""
import numpy as np
import torch


class WeightedPageRankFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, weights, tele, engine):
        x, _ = engine.forward(weights.detach().cpu().numpy(), tele.detach().cpu().numpy())
        ctx.engine = engine
        return torch.from_numpy(x)

    @staticmethod
    def backward(ctx, grad_x):
        gw, gt, _, _ = ctx.engine.backward(grad_x.detach().cpu().numpy().astype(np.float32))
        return torch.from_numpy(gw), torch.from_numpy(gt), None


def weighted_pagerank(weights, tele, engine):
    return WeightedPageRankFn.apply(weights, tele, engine)
