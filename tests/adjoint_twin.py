"""torch complex128 twin of the adjoint form's controlled step (test
infrastructure): W_{n+1} = N(C P(eps_n) K W_n) with V(x) = v4 x^4 + v2 x^2 + v0 +
eps_n x, Caldeira-Leggett order 3 (C) and the normalisation (N) when gamma != 0,
the same model as include/wigner_b200.h's wiga_* form, written with torch.fft
so that autograd gives FP64 reference gradients (with respect to W_0, eps_n and
(v4, v2)).  Its forward step is pinned to the numpy oracle (oracle/wigner2d.py,
the restatement of GPU_Wigner2D_FFT.py:1884-1913) in tests/test_adjoint.py."""
import math

import torch


def shifted_index(n, device):
    k = torch.arange(n, dtype=torch.float64, device=device)
    return torch.where(k < n / 2, k, k - n)


class Twin:
    def __init__(self, n_x, n_p, amp=10., dt=0.005, d_theta=0., d_lambda=0., v4=0.05, v2=-1., v0=0.,
                 hbar=1., mass=1., gamma=0., f_eps=0., device='cpu'):
        self.n_x, self.n_p = n_x, n_p
        dx, dp = 2. * amp / n_x, 2. * amp / n_p
        dth = dlam = 2. * math.pi / (2. * amp)
        jx, jp = shifted_index(n_x, device), shifted_index(n_p, device)
        x, lam = (dx * jx)[None, :], (dlam * jx)[None, :]
        p, th = (dp * jp)[:, None], (dth * jp)[:, None]
        self.dx, self.dp, self.dt, self.hbar = dx, dp, dt, hbar
        self.v4, self.v2 = v4, v2
        self.K = torch.exp(-d_lambda * lam * lam) * torch.exp(-1j * dt * lam * p / mass)
        x_max = dx * (n_x - 1.) / 2.
        w2 = (10. * dx) ** 2
        mask = (1. - torch.exp(-(x - x_max) ** 2 / w2)) * (1. - torch.exp(-(x + x_max) ** 2 / w2))
        self.x = x
        self.u = hbar * th / 2.
        self.R = torch.exp(-d_theta * th * th * dt) * mask
        # V(x - u) - V(x + u) = -8 v4 x u (x^2 + u^2) - 4 v2 x u - 2 eps u
        self.dV4 = -8. * x * self.u * (x * x + self.u * self.u)
        self.dV2 = -4. * x * self.u
        self.dVe = -2. * self.u
        self.gamma = gamma
        g = dt * gamma
        c1, c2, c3 = 2. / 3. * g, g, 2. * g
        self.a1 = 1j * (c1 * c2 / (c1 + c2) if c1 + c2 != 0. else 0.)
        self.a2 = 1j * (c1 + c2)
        self.a3 = 1j * c3
        f = torch.abs(p) if f_eps == 0. else p * p / torch.sqrt(p * p + f_eps)
        self.sfp = torch.where(p >= 0., f, -f).to(torch.complex128)
        self.th = th.to(torch.complex128)

    def P(self, eps, coef=None):
        v4, v2 = (self.v4, self.v2) if coef is None else (coef[0], coef[1])
        dV = v4 * self.dV4 + v2 * self.dV2 + eps * self.dVe
        return self.R * torch.exp(-1j * self.dt * dV / self.hbar)

    def D(self, W):
        return torch.fft.ifft(self.th * torch.fft.fft(self.sfp * W, dim=0), dim=0)

    def step(self, W, eps, coef=None):
        Y = torch.fft.ifft(torch.fft.fft(W, dim=1) * self.K, dim=1)
        A = torch.fft.ifft(torch.fft.fft(Y, dim=0) * self.P(eps, coef), dim=0)
        if self.gamma == 0.:
            return A
        U = A + self.a3 * self.D(A + self.a2 * self.D(A + self.a1 * self.D(A)))
        return U / (U.sum() * self.dx * self.dp)

    def propagate(self, W0, eps_steps, coef=None):
        W = W0
        for n in range(eps_steps.shape[0]):
            W = self.step(W, eps_steps[n], coef)
        return W


def coherent(n, amp, x0, p0, device='cpu'):
    d = 2. * amp / n
    j = shifted_index(n, device) * d
    X, P = j[None, :], j[:, None]
    W = torch.exp(-((X - x0) ** 2 + (P - p0) ** 2))
    return (W / (W.sum() * d * d)).to(torch.complex128)
