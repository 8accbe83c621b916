"""Shared helper of the surrogate tests: the design objective and its
gradient with respect to rho through the NumPy oracle network."""
import numpy as np

from photonfdtd_b200 import surrogate as S


def oracle_value_and_grad(ref, t_mean, t_std, rho):
    """band_objective and its rho-gradient through the NumPy network."""
    import torch
    y = ref.forward(2.0 * rho - 1.0)
    yy = torch.from_numpy(y).requires_grad_(True)
    yd = yy * torch.from_numpy(t_std) + torch.from_numpy(t_mean)
    v = S.band_objective(torch.complex(yd[:, :, 0], yd[:, :, 1]))
    v.sum().backward()
    _, dx = ref.backward(yy.grad.numpy())
    return v.detach().numpy(), 2.0 * dx
