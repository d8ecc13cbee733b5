"""Shared pieces of the CPU oracle (test infrastructure only).

* ``cuda_f``: the reference hands every physical constant to its kernels as
  text through ``'%f'`` formatting (``GPU_Wigner2D_FFT.py:833-842``,
  ``GPU_Dirac2D.py:358-367``), i.e. rounded to 6 decimals.  The oracle's
  ``constants='cuda_%f'`` mode reproduces that; ``'exact'`` keeps full doubles.
* ``shifted_range``: the reference's grids are ``np.linspace`` ranges put through
  ``fftpack.fftshift`` (``GPU_Wigner2D_FFT.py:568-581``,
  ``GPU_Dirac2D.py:328-346``).
* ``eval_expr``: the reference evaluates its C expression strings on the host
  with ``eval(s, np.__dict__, locals())`` and ``pow = np.power`` etc.
  (``GPU_Wigner2D_FFT.py:674-692,1674-1681``).  The oracle evaluates the same
  strings the same way for both host tables and the device-side kernels.
"""
import math
import os

import numpy as np
import scipy.fft as sfft

WORKERS = os.cpu_count() or 1


def cuda_f(v):
    """``float('%f' % v)``: the 6-decimal rounding the reference applies to the
    constants it pastes into kernel source (``GPU_Wigner2D_FFT.py:834``)."""
    return float('%f' % v)


def shifted_range(amplitude, n):
    """``fftshift(linspace(-a, a - 2a/n, n))`` exactly as the reference builds
    its X/P/Theta/Lambda tables (``GPU_Wigner2D_FFT.py:568-581``)."""
    d = 2.0 * amplitude / float(n)
    return np.fft.fftshift(np.linspace(-amplitude, amplitude - d, n))


def kernel_coord(delta, n):
    """Coordinate a reference kernel rebuilds from an array index:
    ``delta*(((k + n/2) % n) - 0.5*n)`` (``GPU_Wigner2D_FFT.py:106-111``)."""
    k = np.arange(n)
    j = (k + n // 2) % n
    return delta * (j - 0.5 * n)


def kernel_coord_int(delta, n):
    """Dirac variant: ``delta*(j - n/2)`` with integer ``j - n/2``
    (``GPU_Dirac2D.py:49-53``)."""
    k = np.arange(n)
    j = (k + n // 2) % n
    return delta * (j - n // 2).astype(np.float64)


def _namespace(extra):
    ns = dict(np.__dict__)
    ns.update(pow=np.power, atan=np.arctan, M_E=np.e, M_PI=np.pi, sqrt=np.sqrt,
              exp=np.exp, fabs=np.fabs, abs=np.abs, cos=np.cos, sin=np.sin,
              tan=np.tan, log=np.log, cosh=np.cosh, sinh=np.sinh, tanh=np.tanh,
              atan2=np.arctan2, floor=np.floor, ceil=np.ceil)
    ns.update(extra)
    return ns


def eval_expr(expr, **variables):
    """Evaluate a C expression string the way the reference's host side does
    (``eval(expr, np.__dict__, locals())`` with ``pow=np.power``)."""
    out = eval(expr, _namespace(variables))
    return out


def eval_expr_like(expr, shape, **variables):
    """``eval_expr`` broadcast to ``shape`` (constant strings such as ``'0.'``
    evaluate to a scalar)."""
    v = np.asarray(eval_expr(expr, **variables), dtype=np.float64)
    return np.broadcast_to(v, shape).astype(np.float64)


def fft(a, axis):
    """Forward DFT, e^{-i}, unnormalised (cuFFT ``CUFFT_FORWARD`` convention,
    ``cufft_wrapper.py:396-397``)."""
    return sfft.fft(a, axis=axis, workers=WORKERS)


def ifft_unnormalised(a, axis):
    """Inverse DFT, e^{+i}, unnormalised (cuFFT ``CUFFT_INVERSE``,
    ``cufft_wrapper.py:399-400``); callers scale by 1/N as the reference does."""
    return sfft.ifft(a, axis=axis, norm='forward', workers=WORKERS)


def fft2(a):
    return sfft.fft2(a, axes=(-2, -1), workers=WORKERS)


def ifft2_unnormalised(a):
    return sfft.ifft2(a, axes=(-2, -1), norm='forward', workers=WORKERS)


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


def is_pow2(n):
    return n > 0 and (n & (n - 1)) == 0 and math.log2(n) == int(math.log2(n))
