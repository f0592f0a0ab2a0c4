"""log L(theta) as a differentiable PyTorch function (d log L / d log theta by the adjoint method).

For optimisers and samplers that work on torch tensors: the forward solve and the adjoint backward
solve both run in the cufsp library (cufsp_likelihood_grad); the gradient is computed with the
value and kept for backward.
"""
from __future__ import annotations

import numpy as np
import torch

from .likelihood import Likelihood


class _LogLikFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, log_theta: torch.Tensor, lik: Likelihood) -> torch.Tensor:
        theta = np.exp(log_theta.detach().cpu().double().numpy())
        ll, g = lik.gradient(theta)
        ctx.save_for_backward(torch.as_tensor(g, dtype=log_theta.dtype, device=log_theta.device))
        return torch.tensor(ll, dtype=log_theta.dtype, device=log_theta.device)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        (g,) = ctx.saved_tensors
        return grad_out * g, None


def log_likelihood(log_theta: torch.Tensor, lik: Likelihood) -> torch.Tensor:
    """log L at rates exp(log_theta) ([n_reactions]); differentiable in log_theta."""
    return _LogLikFn.apply(log_theta, lik)
