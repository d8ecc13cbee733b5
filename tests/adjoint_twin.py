"""torch complex128 twin of the adjoint form's controlled step (test
infrastructure): W_{n+1} = P(eps_n) K W_n with V(x) = v4 x^4 + v2 x^2 + v0 + eps_n x,
the same model as include/wigner_b200.h's wiga_* form, written with torch.fft
so that autograd gives FP64 reference gradients.  Its forward step is pinned to
the numpy oracle (oracle/wigner2d.py, the restatement of
GPU_Wigner2D_FFT.py:1884-1899) in tests/test_adjoint.py."""
import math

import torch


def shifted_index(n, device):
    k = torch.arange(n, dtype=torch.float64, device=device)
    return torch.where(k < n / 2, k, k - n)


class Twin:
    def __init__(self, n_x, n_p, amp=10., dt=0.005, d_theta=0., d_lambda=0., v4=0.05, v2=-1., v0=0.,
                 hbar=1., mass=1., device='cpu'):
        self.n_x, self.n_p = n_x, n_p
        dx, dp = 2. * amp / n_x, 2. * amp / n_p
        dth = dlam = 2. * math.pi / (2. * amp)
        jx, jp = shifted_index(n_x, device), shifted_index(n_p, device)
        x, lam = (dx * jx)[None, :], (dlam * jx)[None, :]
        p, th = (dp * jp)[:, None], (dth * jp)[:, None]
        self.dx, self.dp = dx, dp
        self.K = torch.exp(-d_lambda * lam * lam) * torch.exp(-1j * dt * lam * p / mass)
        x_max = dx * (n_x - 1.) / 2.
        w2 = (10. * dx) ** 2
        mask = (1. - torch.exp(-(x - x_max) ** 2 / w2)) * (1. - torch.exp(-(x + x_max) ** 2 / w2))
        u = hbar * th / 2.
        dV0 = -2. * u * (4. * v4 * x ** 3 + 4. * v4 * x * u * u + 2. * v2 * x)   # V(x-u) - V(x+u), eps = 0
        self.P0 = torch.exp(-d_theta * th * th * dt) * mask * torch.exp(-1j * dt * dV0 / hbar)
        self.dtth = (dt * th).to(torch.complex128)   # eps x adds exp(i eps dt theta)

    def step(self, W, eps):
        Y = torch.fft.ifft(torch.fft.fft(W, dim=1) * self.K, dim=1)
        return torch.fft.ifft(torch.fft.fft(Y, dim=0) * (self.P0 * torch.exp(1j * eps * self.dtth)), dim=0)

    def propagate(self, W0, eps_steps):
        W = W0
        for n in range(eps_steps.shape[0]):
            W = self.step(W, eps_steps[n])
        return W


def coherent(n, amp, x0, p0, device='cpu'):
    d = 2. * amp / n
    j = shifted_index(n, device) * d
    X, P = j[None, :], j[:, None]
    W = torch.exp(-((X - x0) ** 2 + (P - p0) ** 2))
    return (W / (W.sum() * d * d)).to(torch.complex128)
