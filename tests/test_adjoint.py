"""Adjoint (differentiable) FP32 form: wiga_forward / wig_step_adjoint.

CPU: the torch complex128 twin (tests/adjoint_twin.py) is pinned to the numpy
oracle's step (oracle/wigner2d.py, GPU_Wigner2D_FFT.py:1884-1899) and its
autograd gradient to central finite differences.  GPU: the CUDA forward
against the twin, the transpose identity <lam, M x> = <M^H lam, x> of one
adjoint step, the control and initial-state gradients against the twin's
autograd, central finite differences of the CUDA forward, and the 512^2 /
500-step / 50-segment configuration with checkpoints every 50 steps."""
import math

import numpy as np
import pytest
import torch

from adjoint_twin import Twin, coherent
from oracle.wigner2d import WignerOracle, WignerParams


def test_twin_step_matches_oracle():
    n, amp, dt, eps = 64, 10., 0.01, 0.3
    prm = WignerParams(n, n, amp, amp, dt, potential='0.05*pow(x,4) + -1.0*pow(x,2) + 0.3*x',
                       dpotential='0.2*pow(x,3) - 2.0*x + 0.3', d_theta=0.05, d_lambda=0.002,
                       gamma=0., constants='exact')
    orc = WignerOracle(prm)
    tw = Twin(n, n, amp, dt, d_theta=0.05, d_lambda=0.002)
    W = coherent(n, amp, -1.0, 0.5)
    Wo = W.numpy()
    Wt = W
    for k in range(20):
        Wo = orc.step(Wo, k * dt)
        Wt = tw.step(Wt, torch.tensor(eps, dtype=torch.float64))
    err = np.linalg.norm(Wt.numpy() - Wo) / np.linalg.norm(Wo)
    assert err < 1e-12, err


def test_twin_gradient_matches_finite_differences():
    n, amp, dt = 32, 10., 0.01
    tw = Twin(n, n, amp, dt)
    W0 = coherent(n, amp, -1.0, 0.2)
    target = coherent(n, amp, 1.0, 0.0).real
    theta = torch.tensor([0.1, -0.2, 0.05], dtype=torch.float64, requires_grad=True)

    def loss(th):
        W = tw.propagate(W0, th.repeat_interleave(5))
        return (W.real * target).sum() * tw.dx * tw.dp

    L = loss(theta)
    L.backward()
    for i in range(3):
        h = 1e-5
        tp, tm = theta.detach().clone(), theta.detach().clone()
        tp[i] += h
        tm[i] -= h
        fd = (loss(tp) - loss(tm)).item() / (2 * h)
        assert abs(fd - theta.grad[i].item()) < 1e-7 * max(1., abs(fd)), (i, fd, theta.grad[i].item())


# ---------------------------------------------------------------- GPU
def _setup(n, amp=10., dt=0.005, v4=0.05, v2=-1., d_theta=0., d_lambda=0.):
    from pywignercuda_b200.adjoint import WignerControl
    dev = torch.device('cuda')
    prop = WignerControl(n, x_amplitude=amp, dt=dt, v4=v4, v2=v2, d_theta=d_theta, d_lambda=d_lambda)
    tw = Twin(n, n, amp, dt, d_theta=d_theta, d_lambda=d_lambda, v4=v4, v2=v2, device=dev)
    return prop, tw, dev


@pytest.mark.gpu
def test_forward_matches_twin():
    prop, tw, dev = _setup(128, d_theta=0.02, d_lambda=0.001)
    rng = np.random.default_rng(4)
    eps = torch.tensor(rng.normal(0., 0.1, 100), dtype=torch.float64, device=dev)
    W0 = coherent(128, 10., -2.0, 0.0, device=dev)
    W = W0.to(torch.complex64).contiguous()
    prop.forward_raw(W, eps)
    Wt = tw.propagate(W0, eps)
    err = (torch.linalg.norm(W.to(torch.complex128) - Wt) / torch.linalg.norm(Wt)).item()
    assert err < 1e-4, err      # FP32 FFT rounding over 100 steps


@pytest.mark.gpu
def test_adjoint_step_is_the_transpose():
    prop, tw, dev = _setup(256, d_theta=0.02)
    g = torch.Generator(device='cpu').manual_seed(3)
    shape = (256, 256)
    X = torch.complex(torch.randn(shape, generator=g), torch.randn(shape, generator=g)).to(dev)
    L = torch.complex(torch.randn(shape, generator=g), torch.randn(shape, generator=g)).to(dev)
    eps = torch.tensor([0.0, 0.37], dtype=torch.float64, device=dev)
    W = X.contiguous().clone()
    Y = torch.empty((1, 256, 256), dtype=torch.complex64, device=dev)
    prop.forward_raw(W, eps, 1, 1, Y)                  # W = M_1 X
    lam = L.contiguous().clone()
    grad = torch.zeros(2, dtype=torch.float64, device=dev)
    prop.adjoint_step(lam, Y[0], eps, 1, grad)         # lam = M_1^H L
    lhs = (L.to(torch.complex128).conj() * W.to(torch.complex128)).sum().real.item()
    rhs = (lam.to(torch.complex128).conj() * X.to(torch.complex128)).sum().real.item()
    scale = torch.linalg.norm(L.to(torch.complex128)).item() * torch.linalg.norm(X.to(torch.complex128)).item()
    assert abs(lhs - rhs) < 1e-6 * scale, (lhs, rhs, scale)


def _loss_and_grads(prop, tw, dev, n, theta, seg, W0, target, K):
    theta_t = torch.tensor(theta, dtype=torch.float64, device=dev, requires_grad=True)
    W0c = W0.to(torch.complex64).contiguous().requires_grad_(True)
    WT = prop.propagate(W0c, theta_t.repeat_interleave(seg), checkpoint=K)
    L = (WT.real.to(torch.float64) * target).sum() * tw.dx * tw.dp
    L.backward()
    theta_r = torch.tensor(theta, dtype=torch.float64, device=dev, requires_grad=True)
    W0r = W0.detach().clone().requires_grad_(True)
    WTr = tw.propagate(W0r, theta_r.repeat_interleave(seg))
    Lr = (WTr.real * target).sum() * tw.dx * tw.dp
    Lr.backward()
    return L.item(), theta_t.grad, W0c.grad, Lr.item(), theta_r.grad, W0r.grad


@pytest.mark.gpu
def test_gradients_match_twin_autograd():
    n = 128
    prop, tw, dev = _setup(n)
    rng = np.random.default_rng(1)
    theta = rng.normal(0., 0.1, 12)
    W0 = coherent(n, 10., -2.0, 0.0, device=dev)
    target = coherent(n, 10., 1.5, 0.3, device=dev).real
    L, gt, gW, Lr, gtr, gWr = _loss_and_grads(prop, tw, dev, n, theta, 10, W0, target, K=25)
    assert abs(L - Lr) < 1e-4 * abs(Lr), (L, Lr)
    eg = (torch.linalg.norm(gt - gtr) / torch.linalg.norm(gtr)).item()
    assert eg < 1e-3, eg
    eW = (torch.linalg.norm(gW.to(torch.complex128) - gWr) / torch.linalg.norm(gWr)).item()
    assert eW < 1e-3, eW


@pytest.mark.gpu
def test_gradient_matches_finite_differences_of_the_cuda_forward():
    n = 128
    prop, tw, dev = _setup(n)
    rng = np.random.default_rng(2)
    theta = rng.normal(0., 0.1, 6)
    W0 = coherent(n, 10., -2.0, 0.0, device=dev).to(torch.complex64).contiguous()
    target = coherent(n, 10., 1.5, 0.3, device=dev).real

    def loss(th):
        W = W0.clone()
        prop.forward_raw(W, torch.tensor(th, dtype=torch.float64, device=dev).repeat_interleave(10).contiguous())
        return ((W.real.to(torch.float64) * target).sum() * tw.dx * tw.dp).item()

    theta_t = torch.tensor(theta, dtype=torch.float64, device=dev, requires_grad=True)
    WT = prop.propagate(W0.clone().requires_grad_(False), theta_t.repeat_interleave(10), checkpoint=20)
    ((WT.real.to(torch.float64) * target).sum() * tw.dx * tw.dp).backward()
    for i in range(len(theta)):
        h = 1e-4 * max(abs(theta[i]), 1.)
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (loss(tp) - loss(tm)) / (2 * h)
        g = theta_t.grad[i].item()
        # FP32 forward: the difference quotient carries ~1e-7 / h of rounding noise
        assert abs(fd - g) < 2e-2 * abs(g) + 2e-3, (i, fd, g)


@pytest.mark.gpu
def test_control_configuration_512_500_steps():
    """512^2, V = 0.05 x^4 - x^2 + eps(t) x, eps piecewise constant over 50
    segments of 10 steps (default_rng(1), N(0, 0.1)), coherent state at (-2, 0),
    target Gaussian centre from default_rng(2), loss dxdp sum W_T W_target,
    500 steps, checkpoints every 50."""
    n = 512
    prop, tw, dev = _setup(n)
    theta = np.random.default_rng(1).normal(0., 0.1, 50)
    c = np.random.default_rng(2).uniform(-2., 2., 2)
    W0 = coherent(n, 10., -2.0, 0.0, device=dev)
    target = coherent(n, 10., float(c[0]), float(c[1]), device=dev).real
    L, gt, gW, Lr, gtr, gWr = _loss_and_grads(prop, tw, dev, n, theta, 10, W0, target, K=50)
    assert abs(L - Lr) < 1e-3 * abs(Lr) + 1e-6, (L, Lr)
    eg = (torch.linalg.norm(gt - gtr) / torch.linalg.norm(gtr)).item()
    assert eg < 5e-3, eg
