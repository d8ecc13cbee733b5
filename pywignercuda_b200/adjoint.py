"""Adjoint (differentiable) Wigner2D form (``wiga_*`` / ``wig_step_adjoint``
in include/wigner_b200.h).

One grid advanced by the reference's Lie step (``GPU_Wigner2D_FFT.py:1884-1913``)
W_{n+1} = N(C P(eps_n) K W_n) with V(x) = v4 x^4 + v2 x^2 + v0 + eps_n x, where
eps_n is a control per step; with ``gamma`` != 0, C is the Caldeira-Leggett
order-3 step and N the normalisation (identities when undamped).
``WignerControl.propagate`` is a ``torch.autograd.Function``: the forward sweep
keeps a checkpoint of W every ``checkpoint`` steps; the backward sweep
recomputes each segment's records (Y_n = K W_n, and for damped steps the
output before normalisation U_n and its sum s_n) from its checkpoint and runs
the adjoint steps through them, accumulating dL/d eps_n and dL/d(v4, v2) and
returning dL/dW_0.  Gradients follow torch's convention for complex tensors
(dL = Re sum conj(grad) dW).  ``precision='c64'`` keeps the state in complex64
with FP32 transforms, ``'c128'`` in complex128 with FP64 transforms.  No
counterpart in the reference, which has no gradients.
"""
import ctypes

from . import _lib
from ._lib import WigaDesc, check
from .wigner2d import _torch

PRECISIONS = {'c64': _lib.WIGA_PREC_C64, 'c128': _lib.WIGA_PREC_C128}


class WignerControl:
    """A differentiable propagator for one (n_p, n_x) grid on the current CUDA
    device (grids: powers of two in [64, 1024])."""

    def __init__(self, n_x, n_p=None, x_amplitude=10., p_amplitude=None, hbar=1., mass=1., dt=0.005,
                 d_theta=0., d_lambda=0., v4=0.05, v2=-1., v0=0., gamma=0., f_eps=0., precision='c64'):
        torch = _torch()
        lib = _lib.load()
        if precision not in PRECISIONS:
            raise _lib.WignerArgumentError("precision must be 'c64' or 'c128'")
        n_p = int(n_p or n_x)
        self.desc = WigaDesc(abi_version=_lib.ABI_VERSION, n_x=int(n_x), n_p=n_p, precision=PRECISIONS[precision],
                             x_amplitude=float(x_amplitude),
                             p_amplitude=float(p_amplitude if p_amplitude is not None else x_amplitude),
                             hbar=float(hbar), mass=float(mass), dt=float(dt), d_theta=float(d_theta),
                             d_lambda=float(d_lambda), v4=float(v4), v2=float(v2), v0=float(v0),
                             gamma=float(gamma), f_eps=float(f_eps))
        h = ctypes.c_void_p()
        check(lib.wiga_create(ctypes.byref(self.desc), ctypes.byref(h)), 'wiga_create')
        self._handle = h
        self.n_x, self.n_p = int(n_x), n_p
        self.damped = float(gamma) != 0.
        self.dtype = torch.complex128 if precision == 'c128' else torch.complex64
        self.device = torch.cuda.current_device()

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                _lib.load().wiga_destroy(h)
            except Exception:
                pass
            h.value = None

    def set_potential(self, v4, v2, v0=None):
        """Replace the potential coefficients (V = v4 x^4 + v2 x^2 + v0 + eps x)."""
        v0 = self.desc.v0 if v0 is None else float(v0)
        check(_lib.load().wiga_set_potential(self._handle, float(v4), float(v2), v0), 'wiga_set_potential')
        self.desc.v4, self.desc.v2, self.desc.v0 = float(v4), float(v2), v0

    def _check_plane(self, T, what, lead=None):
        shape = (self.n_p, self.n_x) if lead is None else (lead, self.n_p, self.n_x)
        if T.dtype != self.dtype or not T.is_cuda or not T.is_contiguous() or tuple(T.shape) != shape:
            raise _lib.WignerArgumentError('%s must be a contiguous CUDA %s tensor of shape %s'
                                           % (what, str(self.dtype).split('.')[-1], shape))

    def _check_eps(self, eps, n):
        torch = _torch()
        if eps.dtype != torch.float64 or not eps.is_cuda or not eps.is_contiguous() or eps.numel() < n:
            raise _lib.WignerArgumentError('eps must be a contiguous CUDA float64 tensor with one value per step')

    def _check_s(self, s, n):
        torch = _torch()
        if s.dtype != torch.complex128 or not s.is_cuda or not s.is_contiguous() or s.numel() < n:
            raise _lib.WignerArgumentError('s must be a contiguous CUDA complex128 tensor with one value per step')

    def forward_raw(self, W, eps, step0=0, n_steps=None, Y=None, U=None, s=None, stream=None):
        """Advance W in place by n_steps steps from step index step0 (eps[step]
        is used at each step).  Optional records: Y ((n_steps, n_p, n_x))
        receives Y_n = K W_n; damped: U ((n_steps, n_p, n_x)) the output before
        normalisation and s (complex128, indexed by step) its sum dX dP sum U."""
        torch = _torch()
        n_steps = eps.numel() - step0 if n_steps is None else int(n_steps)
        self._check_plane(W, 'W')
        self._check_eps(eps, step0 + n_steps)
        for T, name in ((Y, 'Y'), (U, 'U')):
            if T is not None:
                self._check_plane(T, name, lead=n_steps)
        if s is not None:
            self._check_s(s, step0 + n_steps)
        st = stream if stream is not None else torch.cuda.current_stream(W.device)
        ptr = lambda T: T.data_ptr() if T is not None else None
        check(_lib.load().wiga_forward(self._handle, W.data_ptr(), eps.data_ptr(), int(step0), n_steps, ptr(Y),
                                       ptr(U), ptr(s), st.cuda_stream), 'wiga_forward')
        return W

    def adjoint_step(self, lam, Y_n, eps, step, grad, U_n=None, s=None, stream=None):
        """One adjoint step: lam (dL/dW_{step+1}) becomes dL/dW_step in place;
        grad[step] ((steps, 3) float64) receives dL/d eps_step and the step's
        shares of dL/dv4 and dL/dv2.  Y_n (and, damped, U_n and s) from
        forward_raw's records of that step."""
        torch = _torch()
        self._check_plane(lam, 'lam')
        self._check_plane(Y_n, 'Y_n')
        self._check_eps(eps, step + 1)
        if self.damped:
            if U_n is None or s is None:
                raise _lib.WignerArgumentError('a damped adjoint step needs U_n and s')
            self._check_plane(U_n, 'U_n')
            self._check_s(s, step + 1)
        if grad.dtype != torch.float64 or not grad.is_cuda or not grad.is_contiguous() or grad.numel() < 3 * (step + 1):
            raise _lib.WignerArgumentError('grad must be a contiguous CUDA float64 (steps, 3) tensor')
        st = stream if stream is not None else torch.cuda.current_stream(lam.device)
        ptr = lambda T: T.data_ptr() if T is not None else None
        check(_lib.load().wig_step_adjoint(self._handle, lam.data_ptr(), Y_n.data_ptr(), ptr(U_n), ptr(s),
                                           eps.data_ptr(), int(step), grad.data_ptr(), st.cuda_stream),
              'wig_step_adjoint')

    def adjoint_sweep(self, lam, Y, eps, step0, grad, U=None, s=None, stream=None):
        """The adjoint steps step0 + n - 1 down to step0 (n = Y.shape[0]) in one
        call: lam (dL/dW_{step0+n}) becomes dL/dW_step0 in place and grad[step]
        receives each step's terms, as n calls of adjoint_step would; Y (and,
        damped, U and s) are the segment's records from forward_raw."""
        torch = _torch()
        n = int(Y.shape[0]) if Y.dim() == 3 else 0
        self._check_plane(lam, 'lam')
        self._check_plane(Y, 'Y', lead=n)
        self._check_eps(eps, step0 + n)
        if self.damped:
            if U is None or s is None:
                raise _lib.WignerArgumentError('a damped adjoint sweep needs U and s')
            self._check_plane(U, 'U', lead=n)
            self._check_s(s, step0 + n)
        if grad.dtype != torch.float64 or not grad.is_cuda or not grad.is_contiguous() or grad.numel() < 3 * (step0 + n):
            raise _lib.WignerArgumentError('grad must be a contiguous CUDA float64 (steps, 3) tensor')
        st = stream if stream is not None else torch.cuda.current_stream(lam.device)
        ptr = lambda T: T.data_ptr() if T is not None else None
        check(_lib.load().wiga_adjoint_sweep(self._handle, lam.data_ptr(), Y.data_ptr(), ptr(U), ptr(s),
                                             eps.data_ptr(), int(step0), n, grad.data_ptr(), st.cuda_stream),
              'wiga_adjoint_sweep')

    def propagate(self, W0, eps, coef=None, checkpoint=50):
        """W_T after eps.numel() steps from W0, differentiable in W0, eps and
        (when given) coef = (v4, v2), a float64 tensor whose values replace the
        handle's potential coefficients."""
        return _ControlFn.apply(W0, eps, coef, self, int(checkpoint))


def _make_fn():
    torch = _torch()

    class ControlFn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, W0, eps, coef, prop, K):
            if coef is not None:
                c = coef.detach().double().cpu()
                prop.set_potential(float(c[0]), float(c[1]))
            eps = eps.detach().contiguous()
            T = eps.numel()
            W = W0.detach().to(prop.dtype).contiguous().clone()
            ckpts = []
            for s0 in range(0, T, K):
                ckpts.append(W.clone())
                prop.forward_raw(W, eps, s0, min(K, T - s0))
            ctx.prop, ctx.K, ctx.T = prop, K, T
            ctx.ckpts = ckpts
            ctx.has_coef = coef is not None
            ctx.coef_dtype = coef.dtype if coef is not None else None
            ctx.W0_dtype = W0.dtype
            ctx.save_for_backward(eps)
            return W

        @staticmethod
        def backward(ctx, gW):
            (eps,) = ctx.saved_tensors
            prop, K, T = ctx.prop, ctx.K, ctx.T
            dev = gW.device
            lam = gW.detach().to(prop.dtype).contiguous().clone()
            grad = torch.zeros((T, 3), dtype=torch.float64, device=dev)
            s = torch.zeros(T, dtype=torch.complex128, device=dev) if prop.damped else None
            Y = U = None
            for si in reversed(range(len(ctx.ckpts))):
                s0 = si * K
                n = min(K, T - s0)
                if Y is None or Y.shape[0] != n:
                    Y = torch.empty((n, prop.n_p, prop.n_x), dtype=prop.dtype, device=dev)
                    U = torch.empty_like(Y) if prop.damped else None
                W = ctx.ckpts[si].clone()
                prop.forward_raw(W, eps, s0, n, Y, U, s)
                prop.adjoint_sweep(lam, Y, eps, s0, grad, U, s)
            ctx.ckpts = None
            g_coef = grad[:, 1:].sum(dim=0).to(ctx.coef_dtype) if ctx.has_coef else None
            gW0 = lam.to(ctx.W0_dtype) if ctx.W0_dtype.is_complex else lam.real.to(ctx.W0_dtype)
            return gW0, grad[:, 0].clone(), g_coef, None, None

    return ControlFn


class _LazyFn:
    fn = None

    @classmethod
    def apply(cls, *args):
        if cls.fn is None:
            cls.fn = _make_fn()
        return cls.fn.apply(*args)


_ControlFn = _LazyFn
