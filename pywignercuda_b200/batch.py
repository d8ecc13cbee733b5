"""Batched Wigner2D propagation (``wigb_*`` in include/wigner_b200.h).

Many independent instances -- polynomial potentials V = v4 x^4 + v2 x^2 +
v1 x + v0, kinetic p^2/2m, Caldeira-Leggett damping with f(p) = |p| (or
p^2/sqrt(p^2 + eps)), uneven power-of-two grids in [64, 1024] -- advance
together: one x-pass and one p-pass launch per step over a work list that
spans all instances, the whole run captured once into a CUDA graph, the tile
shape picked by ``autotune``.  The state is the real Wigner function in FP32
(one float per grid point).  ``precision='f32'`` runs every transform and
factor in FP32; ``'mixed'`` runs the kinetic and Moyal transform pairs and
their factors in FP64 (the three dissipator pairs too up to 256-point
columns, in FP32 above) and rounds each FP64 result to the FP32 state
stochastically, so changes smaller than half an FP32 ulp are kept in
expectation instead of being lost every step.  Phase arguments are formed and
range-reduced in FP64; observables are FP64 (Kahan).
The step is the reference's Lie split (``GPU_Wigner2D_FFT.py:1884-1913``)
with exact constants.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import WigbInstance, check, dptr
from .wigner2d import _torch

OBS_NAMES = ('norm', 'x', 'x2', 'p', 'p2', 'xp', 'dV', 'pdV', 'xdV', 'H', 'negative_area')
PRECISIONS = {'f32': 0, 'mixed': 1}


def instance(n_x, n_p=None, x_amplitude=10., p_amplitude=None, hbar=1., mass=1., dt=0.005, gamma=0.,
             d_theta=0., d_lambda=0., v4=0., v2=0.5, v1=0., v0=0., damping_f=0, f_eps=0.5):
    """Descriptor of one batched instance (V = v4 x^4 + v2 x^2 + v1 x + v0)."""
    return dict(n_x=int(n_x), n_p=int(n_p or n_x), x_amplitude=float(x_amplitude),
                p_amplitude=float(p_amplitude if p_amplitude is not None else x_amplitude),
                hbar=float(hbar), mass=float(mass), dt=float(dt), gamma=float(gamma),
                d_theta=float(d_theta), d_lambda=float(d_lambda), v4=float(v4), v2=float(v2),
                v1=float(v1), v0=float(v0), damping_f=int(damping_f), f_eps=float(f_eps))


class WignerBatch:
    def __init__(self, instances, warps=0, precision='f32'):
        torch = _torch()
        lib = _lib.load()
        if precision not in PRECISIONS:
            raise _lib.WignerArgumentError("precision must be 'f32' or 'mixed'")
        self.precision = precision
        self.instances = [dict(d) for d in instances]
        arr = (WigbInstance * len(instances))()
        for a, d in zip(arr, instances):
            for k, v in d.items():
                setattr(a, k, v)
        self._desc = arr
        h = ctypes.c_void_p()
        check(lib.wigb_create(arr, len(instances), int(warps), PRECISIONS[precision], ctypes.byref(h)),
              'wigb_create')
        self._handle = h
        off = (ctypes.c_int64 * (len(instances) + 1))()
        check(lib.wigb_offsets(h, off), 'wigb_offsets')
        self.offsets = np.array(off[:], dtype=np.int64)
        self.total = int(self.offsets[-1])
        self.device = torch.cuda.current_device()
        self.warps = int(warps or 8)

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                _lib.load().wigb_destroy(h)
            except Exception:
                pass
            h.value = None

    # ---- state packing: instance i is a (n_p, n_x) float32 block at offsets[i] (the real
    # Wigner function; the real part of a complex W_init is taken)
    def pack(self, states):
        torch = _torch()
        flat = np.concatenate([np.ascontiguousarray(np.real(s), dtype=np.float32).ravel() for s in states])
        if flat.size != self.total:
            raise _lib.WignerArgumentError('states do not match the batch geometry')
        return torch.from_numpy(flat).to(torch.device('cuda', self.device))

    def unpack(self, W):
        flat = W.detach().cpu().numpy()
        return [flat[self.offsets[i]:self.offsets[i + 1]].reshape(d['n_p'], d['n_x'])
                for i, d in enumerate(self.instances)]

    def _check_W(self, W):
        torch = _torch()
        if W.dtype != torch.float32 or not W.is_cuda or not W.is_contiguous() or W.numel() != self.total:
            raise _lib.WignerArgumentError('W must be the packed contiguous CUDA float32 state')

    def profile(self):
        """(x-pass ms, p-pass ms, steps) of the last run made with profile=True."""
        ms = (ctypes.c_double * 2)()
        n = ctypes.c_int64()
        check(_lib.load().wigb_profile(self._handle, ms, ctypes.byref(n)), 'wigb_profile')
        return ms[0], ms[1], n.value

    def run(self, W, n_prop, t_index0=0, continue_run=False, graph=True, observables=True, stream=None,
            profile=False, flush_l2=False):
        """Advance the packed state W in place; returns obs[count, n_prop+1, 11]
        (sample k before propagation k, the last after the final one).
        t_index0: the index of the first step.  The mixed form rounds its FP64
        results to the FP32 state stochastically, with random words drawn from
        (step index, pass, point): a run is reproducible, and a continued run
        should pass its first step's index to draw fresh words.
        profile=True (with graph=False) times every x-pass and p-pass launch
        (``profile()``); flush_l2=True then also writes a buffer twice the L2
        size before every step, outside the timed launches."""
        torch = _torch()
        self._check_W(W)
        st = stream if stream is not None else torch.cuda.current_stream(W.device)
        flags = ((_lib.WIG_RUN_CONTINUE if continue_run else 0) | (_lib.WIG_RUN_GRAPH if graph else 0)
                 | (_lib.WIG_RUN_PROFILE if profile else 0) | (_lib.WIG_RUN_FLUSH_L2 if flush_l2 else 0))
        obs = np.empty((len(self.instances), n_prop + 1, _lib.WIG_NOBS)) if observables else None
        check(_lib.load().wigb_run(self._handle, W.data_ptr(), t_index0, n_prop, flags,
                                   dptr(obs) if obs is not None else None, st.cuda_stream), 'wigb_run')
        return obs

    def autotune(self, W_scratch, probe_steps=5, stream=None):
        """Time the candidate tile shapes (8, 4, 2 warps per CTA) on W_scratch
        (overwritten) and keep the fastest; returns (warps, {warps: ms})."""
        torch = _torch()
        self._check_W(W_scratch)
        st = stream if stream is not None else torch.cuda.current_stream(W_scratch.device)
        chosen = ctypes.c_int32()
        ms = (ctypes.c_double * 3)()
        check(_lib.load().wigb_autotune(self._handle, W_scratch.data_ptr(), probe_steps, ctypes.byref(chosen),
                                        ms, st.cuda_stream), 'wigb_autotune')
        self.warps = chosen.value
        return chosen.value, {8: ms[0], 4: ms[1], 2: ms[2]}
