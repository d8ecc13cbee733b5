"""Adjoint (differentiable) form: wiga_forward / wig_step_adjoint.

CPU: the torch complex128 twin (tests/adjoint_twin.py) is pinned to the numpy
oracle's step (oracle/wigner2d.py, GPU_Wigner2D_FFT.py:1884-1913), undamped and
with Caldeira-Leggett damping and the normalisation, and its autograd gradients
(W_0, eps_n, v4, v2) to central finite differences.  GPU: the CUDA forward
against the twin in both precisions, the transpose identity of an undamped
step, the gradients against the twin's autograd, and the control configuration
(512^2, 500 steps, eps over 50 segments, checkpoints every 50) in complex128:
dL/d(a, b, eps) against the twin's autograd and against central differences
of the CUDA forward within 1e-6 relative, undamped and damped."""
import numpy as np
import pytest
import torch

from adjoint_twin import Twin, coherent
from oracle.wigner2d import WignerOracle, WignerParams


@pytest.mark.parametrize('gamma', [0., 0.1])
def test_twin_step_matches_oracle(gamma):
    n, amp, dt, eps = 64, 10., 0.01, 0.3
    prm = WignerParams(n, n, amp, amp, dt, potential='0.05*pow(x,4) + -1.0*pow(x,2) + 0.3*x',
                       dpotential='0.2*pow(x,3) - 2.0*x + 0.3', d_theta=0.05, d_lambda=0.002,
                       gamma=gamma, damping='CaldeiraLeggett', fp_damping='fabs(p)', constants='exact')
    orc = WignerOracle(prm)
    tw = Twin(n, n, amp, dt, d_theta=0.05, d_lambda=0.002, gamma=gamma)
    W = coherent(n, amp, -1.0, 0.5)
    Wo = W.numpy()
    Wt = W
    for k in range(20):
        Wo = orc.step(Wo, k * dt)
        Wt = tw.step(Wt, torch.tensor(eps, dtype=torch.float64))
    err = np.linalg.norm(Wt.numpy() - Wo) / np.linalg.norm(Wo)
    assert err < 1e-12, err


@pytest.mark.parametrize('gamma', [0., 0.1])
def test_twin_gradient_matches_finite_differences(gamma):
    n, amp, dt = 32, 10., 0.01
    tw = Twin(n, n, amp, dt, d_theta=0.05, gamma=gamma)
    W0 = coherent(n, amp, -1.0, 0.2)
    target = coherent(n, amp, 1.0, 0.0).real
    theta = torch.tensor([0.1, -0.2, 0.05, 0.05, -1.0], dtype=torch.float64, requires_grad=True)

    def loss(th):
        W = tw.propagate(W0, th[:3].repeat_interleave(5), th[3:])
        return (W.real * target).sum() * tw.dx * tw.dp

    L = loss(theta)
    L.backward()
    for i in range(5):
        h = 1e-5
        tp, tm = theta.detach().clone(), theta.detach().clone()
        tp[i] += h
        tm[i] -= h
        fd = (loss(tp) - loss(tm)).item() / (2 * h)
        assert abs(fd - theta.grad[i].item()) < 1e-7 * max(1., abs(fd)), (i, fd, theta.grad[i].item())


# ---------------------------------------------------------------- GPU
def _setup(n, amp=10., dt=0.005, v4=0.05, v2=-1., d_theta=0., d_lambda=0., gamma=0., precision='c64'):
    from pywignercuda_b200.adjoint import WignerControl
    dev = torch.device('cuda')
    prop = WignerControl(n, x_amplitude=amp, dt=dt, v4=v4, v2=v2, d_theta=d_theta, d_lambda=d_lambda, gamma=gamma,
                         precision=precision)
    tw = Twin(n, n, amp, dt, d_theta=d_theta, d_lambda=d_lambda, v4=v4, v2=v2, gamma=gamma, device=dev)
    return prop, tw, dev


@pytest.mark.gpu
@pytest.mark.parametrize('precision,gamma,bound', [('c64', 0., 1e-4), ('c128', 0., 1e-12), ('c128', 0.1, 1e-12),
                                                   ('c64', 0.1, 1e-4)])
def test_forward_matches_twin(precision, gamma, bound):
    prop, tw, dev = _setup(128, d_theta=0.02, d_lambda=0.001, gamma=gamma, precision=precision)
    rng = np.random.default_rng(4)
    eps = torch.tensor(rng.normal(0., 0.1, 100), dtype=torch.float64, device=dev)
    W0 = coherent(128, 10., -2.0, 0.0, device=dev)
    W = W0.to(prop.dtype).contiguous().clone()     # (W0 itself when the state is complex128)
    prop.forward_raw(W, eps)
    Wt = tw.propagate(W0, eps)
    err = (torch.linalg.norm(W.to(torch.complex128) - Wt) / torch.linalg.norm(Wt)).item()
    assert err < bound, err      # FP32 transforms: their rounding over 100 steps


@pytest.mark.gpu
@pytest.mark.parametrize('precision,bound', [('c64', 1e-6), ('c128', 1e-13)])
def test_adjoint_step_is_the_transpose(precision, bound):
    prop, tw, dev = _setup(256, d_theta=0.02, precision=precision)
    g = torch.Generator(device='cpu').manual_seed(3)
    shape = (256, 256)
    X = torch.complex(torch.randn(shape, generator=g, dtype=torch.float64),
                      torch.randn(shape, generator=g, dtype=torch.float64)).to(dev).to(prop.dtype)
    L = torch.complex(torch.randn(shape, generator=g, dtype=torch.float64),
                      torch.randn(shape, generator=g, dtype=torch.float64)).to(dev).to(prop.dtype)
    eps = torch.tensor([0.0, 0.37], dtype=torch.float64, device=dev)
    W = X.contiguous().clone()
    Y = torch.empty((1, 256, 256), dtype=prop.dtype, device=dev)
    prop.forward_raw(W, eps, 1, 1, Y)                  # W = M_1 X
    lam = L.contiguous().clone()
    grad = torch.zeros((2, 3), dtype=torch.float64, device=dev)
    prop.adjoint_step(lam, Y[0], eps, 1, grad)         # lam = M_1^H L
    lhs = (L.to(torch.complex128).conj() * W.to(torch.complex128)).sum().real.item()
    rhs = (lam.to(torch.complex128).conj() * X.to(torch.complex128)).sum().real.item()
    scale = torch.linalg.norm(L.to(torch.complex128)).item() * torch.linalg.norm(X.to(torch.complex128)).item()
    assert abs(lhs - rhs) < bound * scale, (lhs, rhs, scale)


def _loss_and_grads(prop, tw, dev, theta, seg, coef, W0, target, K):
    """CUDA adjoint and twin autograd gradients of L = dxdp sum Re(W_T) target."""
    theta_t = torch.tensor(theta, dtype=torch.float64, device=dev, requires_grad=True)
    coef_t = torch.tensor(coef, dtype=torch.float64, device=dev, requires_grad=True)
    W0c = W0.detach().to(prop.dtype).contiguous().clone().requires_grad_(True)
    WT = prop.propagate(W0c, theta_t.repeat_interleave(seg), coef_t, checkpoint=K)
    L = (WT.real.to(torch.float64) * target).sum() * tw.dx * tw.dp
    L.backward()
    theta_r = torch.tensor(theta, dtype=torch.float64, device=dev, requires_grad=True)
    coef_r = torch.tensor(coef, dtype=torch.float64, device=dev, requires_grad=True)
    W0r = W0.detach().clone().requires_grad_(True)
    WTr = tw.propagate(W0r, theta_r.repeat_interleave(seg), coef_r)
    Lr = (WTr.real * target).sum() * tw.dx * tw.dp
    Lr.backward()
    return (L.item(), theta_t.grad, coef_t.grad, W0c.grad, Lr.item(), theta_r.grad, coef_r.grad, W0r.grad)


def _rel(a, b):
    return (torch.linalg.norm((a - b).to(torch.complex128)) / torch.linalg.norm(b.to(torch.complex128))).item()


@pytest.mark.gpu
@pytest.mark.parametrize('precision,gamma,bound', [('c64', 0., 1e-3), ('c128', 0., 1e-10), ('c128', 0.1, 1e-10)])
def test_gradients_match_twin_autograd(precision, gamma, bound):
    n = 128
    prop, tw, dev = _setup(n, d_theta=0.05 if gamma else 0., gamma=gamma, precision=precision)
    rng = np.random.default_rng(1)
    theta = rng.normal(0., 0.1, 12)
    W0 = coherent(n, 10., -2.0, 0.0, device=dev)
    target = coherent(n, 10., 1.5, 0.3, device=dev).real
    L, gt, gc, gW, Lr, gtr, gcr, gWr = _loss_and_grads(prop, tw, dev, theta, 10, [0.05, -1.], W0, target, K=25)
    assert abs(L - Lr) < bound * abs(Lr), (L, Lr)
    assert _rel(gt, gtr) < bound, _rel(gt, gtr)
    assert _rel(gc, gcr) < bound, (gc, gcr)
    assert _rel(gW, gWr) < bound, _rel(gW, gWr)


def _control_case(gamma):
    """512^2, V = a x^4 - b x^2 + eps(t) x with a = 0.05, b = 1, eps piecewise
    constant over 50 segments of 10 steps (default_rng(1), N(0, 0.1)), coherent
    state at (-2, 0), target Gaussian centre from default_rng(2), loss
    dxdp sum W_T W_target, 500 steps, checkpoints every 50; damped: gamma and
    D_theta = 2 gamma m kT (kT = 0.5)."""
    n = 512
    prop, tw, dev = _setup(n, gamma=gamma, d_theta=gamma, precision='c128')
    theta = np.random.default_rng(1).normal(0., 0.1, 50)
    c = np.random.default_rng(2).uniform(-2., 2., 2)
    W0 = coherent(n, 10., -2.0, 0.0, device=dev)
    target = coherent(n, 10., float(c[0]), float(c[1]), device=dev).real
    return prop, tw, dev, theta, W0, target


@pytest.mark.gpu
@pytest.mark.parametrize('gamma', [0., 0.1])
def test_control_configuration_gradients_within_1e6(gamma):
    """dL/d(a, b, eps) of the control configuration (complex128 adjoint) against the
    twin's autograd and central differences (h = 1e-4 max(|q|, 1)) of the CUDA
    forward, within 1e-6 relative (the eps gradient as a vector)."""
    prop, tw, dev, theta, W0, target = _control_case(gamma)
    a, b = 0.05, 1.0
    L, gt, gc, gW, Lr, gtr, gcr, gWr = _loss_and_grads(prop, tw, dev, theta, 10, [a, -b], W0, target, K=50)
    assert abs(L - Lr) < 1e-10 * abs(Lr), (L, Lr)
    assert _rel(gt, gtr) < 1e-6, _rel(gt, gtr)
    assert _rel(gc, gcr) < 1e-6, (gc, gcr)
    assert _rel(gW, gWr) < 1e-6, _rel(gW, gWr)
    W0c = W0.detach().to(prop.dtype).contiguous().clone()

    def loss(th, ab):
        prop.set_potential(ab[0], -ab[1])
        W = W0c.clone()
        prop.forward_raw(W, torch.tensor(th, dtype=torch.float64, device=dev).repeat_interleave(10).contiguous())
        return ((W.real * target).sum() * tw.dx * tw.dp).item()

    params = np.concatenate([[a, b], theta])
    g_ad = np.concatenate([[gc[0].item(), -gc[1].item()], gt.cpu().numpy()])   # dL/db = -dL/dv2
    fd = np.empty_like(params)

    def central(i, h):
        pp, pm = params.copy(), params.copy()
        pp[i] += h
        pm[i] -= h
        return (loss(pp[2:], pp[:2]) - loss(pm[2:], pm[:2])) / (2 * h)
    for i in range(params.size):
        # central differences with h = 1e-4 max(|q|, 1), Richardson-extrapolated with h / 2: the
        # h^2 term of a central difference in a (the x^4 coefficient, q = 0.05, relative step
        # 2e-3) is ~1e-4 of the derivative, which the extrapolation removes
        h = 1e-4 * max(abs(params[i]), 1.)
        fd[i] = (4. * central(i, h / 2) - central(i, h)) / 3.
    prop.set_potential(a, -b)
    for i in range(2):
        assert abs(g_ad[i] - fd[i]) < 1e-6 * abs(fd[i]), ('ab'[i], g_ad[i], fd[i])
    e = np.linalg.norm(g_ad[2:] - fd[2:]) / np.linalg.norm(fd[2:])
    assert e < 1e-6, e


@pytest.mark.gpu
def test_complex64_control_gradients_against_twin():
    """The complex64 (FP32 transforms) adjoint on the control configuration:
    measured agreement with the complex128 twin, reported as its bound."""
    prop, tw, dev, theta, W0, target = _control_case(0.)
    from pywignercuda_b200.adjoint import WignerControl
    prop = WignerControl(512, x_amplitude=10., dt=0.005, v4=0.05, v2=-1., precision='c64')
    L, gt, gc, gW, Lr, gtr, gcr, gWr = _loss_and_grads(prop, tw, dev, theta, 10, [0.05, -1.], W0, target, K=50)
    assert abs(L - Lr) < 1e-3 * abs(Lr) + 1e-6, (L, Lr)
    assert _rel(gt, gtr) < 5e-3, _rel(gt, gtr)
    assert _rel(gc, gcr) < 5e-3, (gc, gcr)


@pytest.mark.gpu
@pytest.mark.parametrize('precision,gamma', [('c128', 0.), ('c128', 0.1), ('c64', 0.1)])
def test_adjoint_sweep_equals_steps(precision, gamma):
    """wiga_adjoint_sweep (one call per checkpoint segment, as the autograd backward
    uses it) launches exactly what the step-by-step wig_step_adjoint calls launch:
    the same dL/dW_0 and gradient rows, bit for bit."""
    prop, tw, dev = _setup(128, d_theta=0.02, gamma=gamma, precision=precision)
    n = 12
    eps = torch.tensor(np.random.default_rng(7).normal(0., 0.2, n), dtype=torch.float64, device=dev)
    W = coherent(128, 10., -1.0, 0.5, device=dev).to(prop.dtype).contiguous()
    Y = torch.empty((n, 128, 128), dtype=prop.dtype, device=dev)
    U = torch.empty_like(Y) if gamma else None
    s = torch.zeros(n, dtype=torch.complex128, device=dev) if gamma else None
    prop.forward_raw(W, eps, 0, n, Y, U, s)
    lam0 = coherent(128, 10., 1.0, -0.5, device=dev).to(prop.dtype).contiguous()
    lam_a, lam_b = lam0.clone(), lam0.clone()
    g_a = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    g_b = torch.zeros_like(g_a)
    for k in reversed(range(n)):
        prop.adjoint_step(lam_a, Y[k], eps, k, g_a, U[k] if U is not None else None, s)
    prop.adjoint_sweep(lam_b, Y, eps, 0, g_b, U, s)
    torch.cuda.synchronize()
    assert torch.equal(lam_a, lam_b)
    assert torch.equal(g_a, g_b)
