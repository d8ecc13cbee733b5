"""Adjoint (differentiable) FP32 Wigner2D form (``wiga_*`` / ``wig_step_adjoint``
in include/wigner_b200.h).

One grid advanced by the reference's Lie step (``GPU_Wigner2D_FFT.py:1884-1899``)
W_{n+1} = P(eps_n) K W_n with V(x) = v4 x^4 + v2 x^2 + v0 + eps_n x, where
eps_n is a control per step, and its adjoint.  ``WignerControl.propagate`` is
a ``torch.autograd.Function``: the forward sweep keeps a checkpoint of W every
``checkpoint`` steps; the backward sweep recomputes each segment's
intermediates Y_n = K W_n from its checkpoint and runs the adjoint steps
through it, accumulating dL/d eps_n and returning dL/dW_0.  Gradients follow
torch's convention for complex tensors (dL = Re sum conj(grad) dW).  No
counterpart in the reference, which has no gradients.
"""
import ctypes

from . import _lib
from ._lib import WigaDesc, check
from .wigner2d import _torch


class WignerControl:
    """A differentiable propagator for one (n_p, n_x) complex64 grid on the
    current CUDA device (grids: powers of two in [64, 1024])."""

    def __init__(self, n_x, n_p=None, x_amplitude=10., p_amplitude=None, hbar=1., mass=1., dt=0.005,
                 d_theta=0., d_lambda=0., v4=0.05, v2=-1., v0=0.):
        torch = _torch()
        lib = _lib.load()
        n_p = int(n_p or n_x)
        self.desc = WigaDesc(abi_version=_lib.ABI_VERSION, n_x=int(n_x), n_p=n_p,
                             x_amplitude=float(x_amplitude),
                             p_amplitude=float(p_amplitude if p_amplitude is not None else x_amplitude),
                             hbar=float(hbar), mass=float(mass), dt=float(dt), d_theta=float(d_theta),
                             d_lambda=float(d_lambda), v4=float(v4), v2=float(v2), v0=float(v0))
        h = ctypes.c_void_p()
        check(lib.wiga_create(ctypes.byref(self.desc), ctypes.byref(h)), 'wiga_create')
        self._handle = h
        self.n_x, self.n_p = int(n_x), n_p
        self.device = torch.cuda.current_device()

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                _lib.load().wiga_destroy(h)
            except Exception:
                pass
            h.value = None

    def _check_state(self, W, what):
        torch = _torch()
        if (W.dtype != torch.complex64 or not W.is_cuda or not W.is_contiguous()
                or tuple(W.shape[-2:]) != (self.n_p, self.n_x)):
            raise _lib.WignerArgumentError('%s must be a contiguous CUDA complex64 (n_p, n_x) tensor' % what)

    def _check_eps(self, eps, n):
        torch = _torch()
        if eps.dtype != torch.float64 or not eps.is_cuda or not eps.is_contiguous() or eps.numel() < n:
            raise _lib.WignerArgumentError('eps must be a contiguous CUDA float64 tensor with one value per step')

    def forward_raw(self, W, eps, step0=0, n_steps=None, Y=None, stream=None):
        """Advance W in place by n_steps steps from step index step0 (eps[step]
        is used at each step); Y (optional, (n_steps, n_p, n_x) complex64)
        receives Y_n = K W_n."""
        torch = _torch()
        n_steps = eps.numel() - step0 if n_steps is None else int(n_steps)
        self._check_state(W, 'W')
        self._check_eps(eps, step0 + n_steps)
        if Y is not None:
            if (Y.dtype != torch.complex64 or not Y.is_cuda or not Y.is_contiguous()
                    or tuple(Y.shape) != (n_steps, self.n_p, self.n_x)):
                raise _lib.WignerArgumentError('Y must be a contiguous CUDA complex64 (n_steps, n_p, n_x) tensor')
        st = stream if stream is not None else torch.cuda.current_stream(W.device)
        check(_lib.load().wiga_forward(self._handle, W.data_ptr(), eps.data_ptr(), int(step0), n_steps,
                                       Y.data_ptr() if Y is not None else None, st.cuda_stream), 'wiga_forward')
        return W

    def adjoint_step(self, lam, Y_n, eps, step, grad, stream=None):
        """One adjoint step: lam (dL/dW_{step+1}) becomes dL/dW_step in place;
        grad[step] receives dL/d eps_step.  Y_n: Y of that step."""
        torch = _torch()
        self._check_state(lam, 'lam')
        self._check_state(Y_n, 'Y_n')
        self._check_eps(eps, step + 1)
        if grad.dtype != torch.float64 or not grad.is_cuda or grad.numel() <= step:
            raise _lib.WignerArgumentError('grad must be a CUDA float64 tensor with one value per step')
        st = stream if stream is not None else torch.cuda.current_stream(lam.device)
        check(_lib.load().wig_step_adjoint(self._handle, lam.data_ptr(), Y_n.data_ptr(), eps.data_ptr(),
                                           int(step), grad.data_ptr(), st.cuda_stream), 'wig_step_adjoint')

    def propagate(self, W0, eps, checkpoint=50):
        """W_T after eps.numel() steps from W0, differentiable in W0 and eps."""
        return _ControlFn.apply(W0, eps, self, int(checkpoint))


def _make_fn():
    torch = _torch()

    class ControlFn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, W0, eps, prop, K):
            eps = eps.detach().contiguous()
            T = eps.numel()
            W = W0.detach().contiguous().clone()
            ckpts = []
            for s0 in range(0, T, K):
                ckpts.append(W.clone())
                prop.forward_raw(W, eps, s0, min(K, T - s0))
            ctx.prop, ctx.K, ctx.T = prop, K, T
            ctx.ckpts = ckpts
            ctx.save_for_backward(eps)
            return W

        @staticmethod
        def backward(ctx, gW):
            (eps,) = ctx.saved_tensors
            prop, K, T = ctx.prop, ctx.K, ctx.T
            lam = gW.detach().to(torch.complex64).contiguous().clone()
            grad = torch.zeros(T, dtype=torch.float64, device=lam.device)
            Y = None
            for si in reversed(range(len(ctx.ckpts))):
                s0 = si * K
                n = min(K, T - s0)
                if Y is None or Y.shape[0] != n:
                    Y = torch.empty((n, prop.n_p, prop.n_x), dtype=torch.complex64, device=lam.device)
                W = ctx.ckpts[si].clone()
                prop.forward_raw(W, eps, s0, n, Y)
                for k in reversed(range(n)):
                    prop.adjoint_step(lam, Y[k], eps, s0 + k, grad)
            ctx.ckpts = None
            return lam, grad, None, None

    return ControlFn


class _LazyFn:
    fn = None

    @classmethod
    def apply(cls, *args):
        if cls.fn is None:
            cls.fn = _make_fn()
        return cls.fn.apply(*args)


_ControlFn = _LazyFn
