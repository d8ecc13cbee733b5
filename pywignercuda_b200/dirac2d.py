"""Drop-in Dirac2D propagator: ``GPU_Dirac2D`` (``GPU_Dirac2D.py:288-1133``).

An instance subclass sets ``mass``, ``c``, ``hBar``, ``Potential_0_String`` ..
``Potential_3_String`` (C expressions in t, x, y) and ``fileName``, calls
``GPU_Dirac2D.__init__(self, gridDIM, amplitude, dt, timeSteps, skipFrames,
frameSaveMode)``, sets ``Psi_init`` (array of 4 FFT-shifted (Y, X) spinor
components) and calls ``Run()``, which returns 0 and leaves ``Psi_end``,
``timeRange``, ``X_average``, ``Y_average``, ``Alpha1_average``,
``Alpha2_average``, ``Beta_average``, ``KEnergy_average`` and
``Potential_0_average`` (``:1117-1131``), plus ``Px_average`` / ``Py_average``
(momentum-space averages after ``Normalize_P``; no reference counterpart),
``NormKept_average`` (fraction of the norm the absorbing boundary kept in the
preceding step) and ``frames`` (spinor or density every ``skipFrames`` steps,
``save_Spinor`` / ``save_Density`` :703-737).  With ``fileName`` set, the run
writes the reference's file layout (``frames.py``).

The propagation runs on the GPU through ``libwigner_b200.so``; device memory
and the stream come from PyTorch.  There is no CPU path.
"""
import ctypes

import numpy as np
from scipy.special import eval_genlaguerre, eval_laguerre, eval_legendre

from . import _lib, frames
from ._lib import DiracDesc, check, dptr
from .wigner2d import _torch


class GPU_Dirac2D:
    constants_mode = _lib.CONST_CUDA_F

    def __init__(self, gridDIM, amplitude, dt, timeSteps, skipFrames=1, frameSaveMode='Density'):
        self._set_grids(gridDIM, amplitude)
        self.timeSteps = timeSteps
        self.skipFrames = skipFrames
        self.frameSaveMode = frameSaveMode
        self.dt = dt
        if not hasattr(self, 'hBar'):
            self.hBar = 1.
        for name in ('mass', 'c'):
            if not hasattr(self, name):
                raise _lib.WignerArgumentError('set self.%s before GPU_Dirac2D.__init__' % name)
        for k in range(4):
            if not hasattr(self, 'Potential_%d_String' % k):
                setattr(self, 'Potential_%d_String' % k, '0.')
        self._build()

    def _set_grids(self, gridDIM, amplitude):
        """Shifted x, y and momentum grids (GPU_Dirac2D.py:306-352); host only."""
        X_amplitude, Y_amplitude = amplitude
        X_gridDIM, Y_gridDIM = gridDIM
        self.dX = 2. * X_amplitude / float(X_gridDIM)
        self.dY = 2. * Y_amplitude / float(Y_gridDIM)
        self.X_amplitude, self.Y_amplitude = X_amplitude, Y_amplitude
        self.X_gridDIM, self.Y_gridDIM = X_gridDIM, Y_gridDIM
        self.min_X, self.min_Y = -X_amplitude, -Y_amplitude
        rangeX = np.linspace(-X_amplitude, X_amplitude - self.dX, X_gridDIM)
        rangeY = np.linspace(-Y_amplitude, Y_amplitude - self.dY, Y_gridDIM)
        self.X = np.fft.fftshift(rangeX)[np.newaxis, :]
        self.Y = np.fft.fftshift(rangeY)[:, np.newaxis]
        Px_amplitude = np.pi / self.dX
        self.dPx = 2 * Px_amplitude / self.X_gridDIM
        Px_range = np.linspace(-Px_amplitude, Px_amplitude - self.dPx, self.X_gridDIM)
        Py_amplitude = np.pi / self.dY
        self.dPy = 2 * Py_amplitude / self.Y_gridDIM
        Py_range = np.linspace(-Py_amplitude, Py_amplitude - self.dPy, self.Y_gridDIM)
        self.Px = np.fft.fftshift(Px_range)[np.newaxis, :]
        self.Py = np.fft.fftshift(Py_range)[:, np.newaxis]

    def _build(self):
        lib = _lib.load()
        self._tabs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                      (self.X[0], self.Y[:, 0], self.Px[0], self.Py[:, 0])]
        d = DiracDesc()
        d.abi_version = _lib.ABI_VERSION
        d.n_x, d.n_y = int(self.X_gridDIM), int(self.Y_gridDIM)
        d.constants = self.constants_mode
        d.precision = _lib.PREC_C128
        d.x_amplitude, d.y_amplitude = float(self.X_amplitude), float(self.Y_amplitude)
        d.mass, d.c, d.hbar, d.dt = float(self.mass), float(self.c), float(self.hBar), float(self.dt)
        self._strings = [str(getattr(self, 'Potential_%d_String' % k)).encode() for k in range(4)]
        d.a0, d.a1, d.a2, d.a3 = self._strings
        d.x_table, d.y_table, d.px_table, d.py_table = [dptr(t) for t in self._tabs]
        coefs = getattr(self, 'coefficients', None)
        if coefs is not None:
            for i, v in enumerate(coefs):
                d.coef[i] = float(v)
        self._desc = d
        torch = _torch()
        self._device = torch.cuda.current_device()
        h = ctypes.c_void_p()
        check(lib.dirac_create(d, h), 'dirac_create')
        self._handle = h

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                _lib.load().dirac_destroy(h)
            except Exception:
                pass
            h.value = None

    # ------------------------------------------------------------------ spinors (:419-497)
    def Spinor_Particle_SpinUp(self, p_init, modulation_Function):
        px, py = p_init
        rho = np.exp(1j * self.X * px + 1j * self.Y * py) * modulation_Function(self.X, self.Y)
        p0 = np.sqrt(px * px + py * py + (self.mass * self.c) ** 2)
        return np.array([rho * (p0 + self.mass * self.c), rho * 0., rho * 0., rho * (px + 1j * py)])

    def Spinor_Particle_SpinDown(self, p_init, modulation_Function):
        px, py = p_init
        rho = np.exp(1j * self.X * px + 1j * self.Y * py) * modulation_Function(self.X, self.Y)
        p0 = np.sqrt(px * px + py * py + (self.mass * self.c) ** 2)
        return np.array([rho * 0., rho * (p0 + self.mass * self.c), rho * (px - 1j * py), rho * 0.])

    def Spinor_AntiParticle_SpinDown(self, p_init, modulation_Function):
        px, py = p_init
        rho = np.exp(1j * self.X * px + 1j * self.Y * py) * modulation_Function(self.X, self.Y)
        p0 = -np.sqrt(px * px + py * py + (self.mass * self.c) ** 2)
        return -1j * np.array([rho * 0., rho * (px + 1j * py), rho * (p0 - self.mass * self.c), rho * 0.])

    def Spinor_AntiParticle_SpinUp(self, p_init, modulation_Function):
        px, py = p_init
        rho = np.exp(1j * self.X * px + 1j * self.Y * py) * modulation_Function(self.X, self.Y)
        p0 = -np.sqrt(px * px + py * py + (self.mass * self.c) ** 2)
        return -1j * np.array([rho * (px - 1j * py), rho * 0., rho * 0., rho * (p0 - self.mass * self.c)])

    def Boost(self, p1, p2):
        p0 = np.sqrt((self.mass * self.c) ** 2 + p1 ** 2 + p2 ** 2)
        B00 = self.mass * self.c + p0
        p_Plus, p_Minus = p1 + 1j * p2, p1 - 1j * p2
        return np.array([[B00, 0., 0., p_Minus], [0., B00, p_Plus, 0.], [0., p_Minus, B00, 0.],
                         [p_Plus, 0., 0., B00]])

    def LandauLevelSpinor(self, B, n, x, y, type=1):
        def energy(n):
            return np.sqrt((self.mass * self.c ** 2) ** 2 + 2 * B * self.c * self.hBar * n)
        K = B * ((self.X - x) ** 2 + (self.Y - y) ** 2) / (4. * self.c * self.hBar)
        psi1 = np.exp(-K) * (energy(n) + self.mass * self.c ** 2) * eval_laguerre(n, 2 * K)
        psi3 = np.exp(-K) * (energy(n) - self.mass * self.c ** 2) * eval_laguerre(n, 2 * K)
        if n > 0:
            psi2 = 1j * np.exp(-K) * (self.X - x + 1j * (self.Y - y)) * eval_genlaguerre(n - 1, 1, 2 * K)
        else:
            psi2 = 0. * K
        psi4 = psi2
        if type == 1:
            spinor = np.array([psi1, 0 * psi2, 0 * psi3, psi4])
        elif type == 2:
            spinor = np.array([0 * psi1, psi2, psi3, 0 * psi4])
        else:
            raise _lib.WignerArgumentError('type spinor must be 1 or 2')
        return spinor / self.Norm(spinor)

    def FilterElectrons(self, sign, Psi):
        """Electron (sign=1) / positron (sign=-1) projection in momentum space (:641-701)."""
        px, py = self.c * self.Px, self.c * self.Py
        m, c = self.mass, self.c
        energy = np.sqrt((m * c ** 2) ** 2 + px ** 2 + py ** 2)
        a = sign * m * c ** 2 / energy
        f = [np.fft.fft2(p) for p in Psi]
        out = [(1. + a) * f[0] + sign * (px - 1j * py) / energy * f[3],
               (1. + a) * f[1] + sign * (px + 1j * py) / energy * f[2],
               sign * (px - 1j * py) / energy * f[1] + (1. - a) * f[2],
               sign * (px + 1j * py) / energy * f[0] + (1. - a) * f[3]]
        return np.array([np.fft.ifft2(o) for o in out])

    def Density_From_Spinor(self, Psi):
        return sum(np.abs(Psi[k]) ** 2 for k in range(4))

    def Norm(self, Psi):
        norm = sum(np.sum(np.abs(Psi[k]) ** 2) for k in range(4))
        return np.sqrt(norm * self.dX * self.dY)

    # ------------------------------------------------------------------ run
    def propagate(self, psi, n_steps, t_index0=0, stream=None):
        """Advance the device spinor ``psi`` (torch complex128 (4, Y, X), in place)
        by ``n_steps`` propagations at t = dt*(t_index0 + k), k = 1..n_steps;
        returns the (n_steps, 10) samples (x, y, alpha1, alpha2, beta, K, A0, px, py,
        norm_kept)."""
        torch = _torch()
        if psi.dtype != torch.complex128 or not psi.is_cuda or not psi.is_contiguous() or \
                tuple(psi.shape) != (4, self.Y_gridDIM, self.X_gridDIM):
            raise _lib.WignerArgumentError('psi must be a contiguous CUDA complex128 tensor (4, Y, X)')
        obs = np.empty((n_steps, _lib.DIRAC_NOBS))
        st = stream if stream is not None else torch.cuda.current_stream(psi.device)
        check(_lib.load().dirac_run(self._handle, psi.data_ptr(), t_index0, n_steps, dptr(obs),
                                    st.cuda_stream), 'dirac_run')
        return obs

    def Run(self):
        torch = _torch()
        P0 = np.ascontiguousarray(np.asarray(self.Psi_init), dtype=np.complex128)
        if P0.shape != (4, self.Y_gridDIM, self.X_gridDIM):
            raise _lib.WignerArgumentError('Psi_init must have shape (4, Y_gridDIM, X_gridDIM)')
        self.Psi1_init, self.Psi2_init, self.Psi3_init, self.Psi4_init = P0
        dev = torch.device('cuda', self._device)
        n = int(self.timeSteps)
        skip = max(int(self.skipFrames), 1)
        fileName = getattr(self, 'fileName', '')
        sink = None
        if fileName:                                       # :974-1009
            sink = frames.open_write(fileName)
            frames.dirac_header(sink, self)
        emit = frames.dirac_frame(self.frameSaveMode) if sink is not None else \
            frames.dirac_frame_nosink(self.frameSaveMode)
        self.frames = {0: np.array(emit(sink, 0, P0), copy=True)}   # the initial spinor (:1030-1033)
        obs = np.empty((n, _lib.DIRAC_NOBS))
        with torch.cuda.device(dev):
            psi = torch.from_numpy(P0.copy()).to(dev)
            writer = frames.FrameWriter(psi, sink, emit, keep=self.frames)
            try:
                t = 0
                while t < n:
                    nxt = min(n, (t // skip + 1) * skip)
                    obs[t:nxt] = self.propagate(psi, nxt - t, t_index0=t)
                    t = nxt
                    if t % skip == 0:                      # after step t (:1105-1111)
                        writer.capture(t, psi)
                self.Psi_end = psi.cpu().numpy()
            finally:
                writer.close()
        if sink is not None:
            sink.close()
        self.Psi_init = P0
        self.timeRange = np.arange(1, n + 1)
        (self.X_average, self.Y_average, self.Alpha1_average, self.Alpha2_average, self.Beta_average,
         self.KEnergy_average, self.Potential_0_average, self.Px_average, self.Py_average,
         self.NormKept_average) = [obs[:, k].copy() for k in range(10)]
        return 0

    def load_Density(self, n, fileName=None):
        """The density frame of step ``n`` (``load_Density`` :739-749)."""
        return frames.read(fileName or self.fileName, '/' + str(n))

    def load_Spinor(self, n, fileName=None):
        """The spinor frame of step ``n`` (``load_Spinor`` :751-769)."""
        f = frames.open_read(fileName or self.fileName)
        try:
            return np.array([np.array(f['%d/real/%d' % (k, n)][...]) + 1j * np.array(f['%d/imag/%d' % (k, n)][...])
                             for k in range(1, 5)])
        finally:
            f.close()
