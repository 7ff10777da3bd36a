"""Differentiable exact log-probabilities: d log2 Pr(b) / d(rotation angles) through the adjoint DP sweep.

The amplitude of a string is multilinear in the per-qubit matrices, <b|psi> = 2^{-n/2} Z(b) with
Z(b) = sum_x prod_j M_j[b_j, x_j] (-1)^{x^T A x} (amp.py), and a rotation layer enters only through
M_j = U3(theta_j) M0_j, where M0_j = U_j^dag is the graph form's local Clifford (the tail without rotations).
The GPU computes Z(b) and dZ/dM_k[b_k][x] for every step k in one forward and one adjoint sweep (libgsb
gsb_grad_run); ``LogProb`` wraps that as a torch.autograd.Function of the step matrices, and ``step_matrices``
builds those matrices from the angles with torch ops, so autograd carries the gradient to theta.

  log2 Pr(b) = log2 |Z|^2 - n,   d log2 Pr = (2 / ln 2) Re( sum_{k,x} (dZ/dM_k[b_k][x] / Z) dM_k[b_k][x] ),
so the gradient torch expects for the complex input M (dL/dRe M + i dL/dIm M) is (2 / ln 2) conj(dZ/dM / Z).
"""
import math

import numpy as np
import torch

import gsb


def u3(theta):
    """U3(theta, phi, lambda) for rows of `theta` [..., 3] (amp.u3_matrix), complex128, differentiable."""
    th, ph, la = theta[..., 0], theta[..., 1], theta[..., 2]
    c = torch.cos(th / 2).to(torch.complex128)
    s = torch.sin(th / 2).to(torch.complex128)
    eph = torch.exp(1j * ph.to(torch.float64))
    ela = torch.exp(1j * la.to(torch.float64))
    row0 = torch.stack([c, -ela * s], dim=-1)
    row1 = torch.stack([eph * s, eph * ela * c], dim=-1)
    return torch.stack([row0, row1], dim=-2)


def step_matrices(theta, M0, step_vertices):
    """M_k = U3(theta_v) M0_v for the vertex v eliminated at step k: [ns, 2, 2] complex128 (differentiable in theta).
    theta: [n, 3] real tensor; M0: [n, 2, 2] complex (numpy or tensor)."""
    M0t = torch.as_tensor(np.asarray(M0), dtype=torch.complex128, device=theta.device)
    Mq = u3(theta.to(torch.float64)) @ M0t
    return Mq[torch.as_tensor(step_vertices, device=theta.device)]


class LogProb(torch.autograd.Function):
    """log2 Pr(b_s) for the rows of `bits` (step order), differentiable in the step matrices M [ns, 2, 2]."""

    @staticmethod
    def forward(ctx, M, bits, sweep):
        z, dz = sweep.run(M.detach().cpu().numpy(), bits)
        lp = np.log2(np.abs(z) ** 2) - sweep.n
        g = dz / z[:, None, None]                    # (1/Z) dZ/dM_k[b_k][x]
        ctx.save_for_backward(torch.from_numpy(g), torch.from_numpy(np.ascontiguousarray(bits, np.int64)))
        ctx.device = M.device
        return torch.from_numpy(lp).to(M.device)

    @staticmethod
    def backward(ctx, grad_lp):
        g, bits = ctx.saved_tensors
        w = grad_lp.detach().to("cpu", torch.float64)[:, None, None] * (2 / math.log(2)) * torch.conj(g)
        G = torch.zeros(g.shape[1], 2, 2, dtype=torch.complex128)
        for b in (0, 1):
            G[:, b, :] = (w * (bits == b)[:, :, None]).sum(0)
        return G.to(ctx.device), None, None


def log2_prob(theta, M0, step_vertices, bits, sweep):
    """log2 Pr(b) [nstr] for rotation angles theta [n, 3]; differentiable in theta."""
    return LogProb.apply(step_matrices(theta, M0, step_vertices), bits, sweep)
