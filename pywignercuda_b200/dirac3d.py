"""Drop-in Dirac3D propagator: ``GPU_Dirac3D`` (``GPU_Dirac3D.py:616-1500``).

An instance subclass sets ``mass``, ``c``, ``hBar``, ``Potential_0_String`` ..
``Potential_3_String`` (C expressions in t, x, y, z), ``fileName`` and
``Compute_Ehrenfest_P``, calls ``GPU_Dirac3D.__init__(self, gridDIM, amplitude,
dt, timeSteps, skipFrames, frameSaveMode)`` with 3-tuples, sets ``Psi_init``
(array of 4 FFT-shifted (Z, Y, X) spinor components) and calls ``Run()``, which
returns 0 and leaves ``Psi_end``, ``timeRange``, ``X_average``, ``Y_average``,
``Z_average``, ``Alpha1_average``, ``Alpha2_average``, ``Alpha3_average``,
``Potential_0_average`` and, with ``Compute_Ehrenfest_P`` (default True),
``Px_average``, ``Py_average``, ``Pz_average`` and ``K_Energy_average``
(``:1479-1492``), plus ``Norm_average`` (sum |psi|^2 dX dY dZ of each sample)
and ``frames`` (the density, or in ``'Spinor'`` mode the z = 0 and y = 0 slices
of ``save_Spinor_SliceYZ``, every ``skipFrames`` steps).  With ``fileName`` set
the run writes the reference's file layout (``frames.py``).

Differences from the reference: the 3-D transform is the transform of the
(Z, Y, X) arrays as laid out (the reference's plan ``cufftPlanMany(3, [X, Y, Z])``
agrees only when X == Z); the file's ``z_gridDIM`` / ``z_amplitude`` / ``dz`` are
the z values (the reference writes the y values there, :1279-1288); grids are
powers of two in [16, 512] per axis and ``mass`` must be > 0.

The propagation runs on the GPU through ``libwigner_b200.so``; device memory
and the stream come from PyTorch.  There is no CPU path.
"""
import ctypes

import numpy as np

from . import _lib, frames
from ._lib import Dirac3Desc, check, dptr
from .wigner2d import _torch


class GPU_Dirac3D:
    constants_mode = _lib.CONST_CUDA_F

    def __init__(self, gridDIM, amplitude, dt, timeSteps, skipFrames=1, frameSaveMode='Density'):
        X_amplitude, Y_amplitude, Z_amplitude = amplitude
        X_gridDIM, Y_gridDIM, Z_gridDIM = gridDIM
        self.dX = 2. * X_amplitude / float(X_gridDIM)
        self.dY = 2. * Y_amplitude / float(Y_gridDIM)
        self.dZ = 2. * Z_amplitude / float(Z_gridDIM)
        self.X_amplitude, self.Y_amplitude, self.Z_amplitude = X_amplitude, Y_amplitude, Z_amplitude
        self.X_gridDIM, self.Y_gridDIM, self.Z_gridDIM = X_gridDIM, Y_gridDIM, Z_gridDIM
        self.min_X, self.min_Y = -X_amplitude, -Y_amplitude
        self.timeSteps = timeSteps
        self.skipFrames = skipFrames
        self.frameSaveMode = frameSaveMode
        rangeX = np.linspace(-X_amplitude, X_amplitude - self.dX, X_gridDIM)
        rangeY = np.linspace(-Y_amplitude, Y_amplitude - self.dY, Y_gridDIM)
        rangeZ = np.linspace(-Z_amplitude, Z_amplitude - self.dZ, Z_gridDIM)
        self.X = np.fft.fftshift(rangeX)[np.newaxis, np.newaxis, :]
        self.Y = np.fft.fftshift(rangeY)[np.newaxis, :, np.newaxis]
        self.Z = np.fft.fftshift(rangeZ)[:, np.newaxis, np.newaxis]
        # momentum grids (the kernels rebuild p from dPx (j - N/2); these are for host use)
        self.dPx = 2 * (np.pi / self.dX) / X_gridDIM
        self.dPy = 2 * (np.pi / self.dY) / Y_gridDIM
        self.dPz = 2 * (np.pi / self.dZ) / Z_gridDIM
        self.Px = np.fft.fftshift(np.linspace(-np.pi / self.dX, np.pi / self.dX - self.dPx,
                                              X_gridDIM))[np.newaxis, np.newaxis, :]
        self.Py = np.fft.fftshift(np.linspace(-np.pi / self.dY, np.pi / self.dY - self.dPy,
                                              Y_gridDIM))[np.newaxis, :, np.newaxis]
        self.Pz = np.fft.fftshift(np.linspace(-np.pi / self.dZ, np.pi / self.dZ - self.dPz,
                                              Z_gridDIM))[:, np.newaxis, np.newaxis]
        self.dt = dt
        if not hasattr(self, 'hBar'):
            self.hBar = 1.
        for name in ('mass', 'c'):
            if not hasattr(self, name):
                raise _lib.WignerArgumentError('set self.%s before GPU_Dirac3D.__init__' % name)
        for k in range(4):
            if not hasattr(self, 'Potential_%d_String' % k):
                setattr(self, 'Potential_%d_String' % k, '0.')
        self._build()

    def _build(self):
        lib = _lib.load()
        d = Dirac3Desc()
        d.abi_version = _lib.ABI_VERSION
        d.n_x, d.n_y, d.n_z = int(self.X_gridDIM), int(self.Y_gridDIM), int(self.Z_gridDIM)
        d.constants = self.constants_mode
        d.precision = _lib.PREC_C128
        d.x_amplitude, d.y_amplitude = float(self.X_amplitude), float(self.Y_amplitude)
        d.z_amplitude = float(self.Z_amplitude)
        d.mass, d.c, d.hbar, d.dt = float(self.mass), float(self.c), float(self.hBar), float(self.dt)
        self._strings = [str(getattr(self, 'Potential_%d_String' % k)).encode() for k in range(4)]
        d.a0, d.a1, d.a2, d.a3 = self._strings
        coefs = getattr(self, 'coefficients', None)
        if coefs is not None:
            for i, v in enumerate(coefs):
                d.coef[i] = float(v)
        self._desc = d
        torch = _torch()
        self._device = torch.cuda.current_device()
        h = ctypes.c_void_p()
        check(lib.dirac3_create(d, h), 'dirac3_create')
        self._handle = h

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                _lib.load().dirac3_destroy(h)
            except Exception:
                pass
            h.value = None

    # ------------------------------------------------------------------ spinors (:787-856)
    def _plane_wave(self, p_init, modulation_Function, sign=1.):
        px, py, pz = p_init
        rho = np.exp(sign * 1j * (px * self.X + py * self.Y + pz * self.Z)) * \
            modulation_Function(self.X, self.Y, self.Z)
        p0 = np.sqrt(px * px + py * py + pz * pz + (self.mass * self.c) ** 2)
        return rho, px, py, pz, p0

    def Spinor_Particle_SpinUp(self, p_init, modulation_Function):
        rho, px, py, pz, p0 = self._plane_wave(p_init, modulation_Function)
        return np.array([rho * (p0 + self.mass * self.c), rho * 0., rho * pz, rho * (px + 1j * py)])

    def Spinor_Particle_SpinDown(self, p_init, modulation_Function):
        rho, px, py, pz, p0 = self._plane_wave(p_init, modulation_Function)
        return np.array([rho * 0., rho * (p0 + self.mass * self.c), rho * (px - 1j * py), rho * (-pz)])

    def Spinor_AntiParticle_SpinUp(self, p_init, modulation_Function):
        rho, px, py, pz, p0 = self._plane_wave(p_init, modulation_Function, -1.)
        return -1j * np.array([rho * (px - 1j * py), -rho * pz, rho * 0., rho * (p0 - self.mass * self.c)])

    def Spinor_AntiParticle_SpinDown(self, p_init, modulation_Function):
        rho, px, py, pz, p0 = self._plane_wave(p_init, modulation_Function, -1.)
        return -1j * np.array([rho * pz, rho * (px + 1j * py), rho * (p0 - self.mass * self.c), rho * 0.])

    def Boost(self, p1, p2):
        p0 = np.sqrt((self.mass * self.c) ** 2 + p1 ** 2 + p2 ** 2)
        B00 = self.mass * self.c + p0
        p_Plus, p_Minus = p1 + 1j * p2, p1 - 1j * p2
        return np.array([[B00, 0., 0., p_Minus], [0., B00, p_Plus, 0.], [0., p_Minus, B00, 0.],
                         [p_Plus, 0., 0., B00]])

    def FilterElectrons(self, sign):
        """Keep electrons (sign = 1) or positrons (sign = -1) of ``Psi_init`` by the
        momentum-space projector (:956-1019), in place."""
        def grid(n, amp):
            mn = np.pi * n / (-2 * amp)
            dp = 2 * np.abs(mn) / n
            return np.fft.fftshift(np.linspace(mn, np.abs(mn) - dp, n))
        px = grid(self.X_gridDIM, self.X_amplitude)[np.newaxis, np.newaxis, :]
        py = grid(self.Y_gridDIM, self.Y_amplitude)[np.newaxis, :, np.newaxis]
        pz = grid(self.Z_gridDIM, self.Z_amplitude)[:, np.newaxis, np.newaxis]
        m, c = self.mass, self.c
        sqrtp = sign * 2 * np.sqrt(m * m * c ** 4 + c * c * px * px + c * c * py * py + c * c * pz * pz)
        aa = sign * m * c * c / sqrtp
        bb = sign * (px / sqrtp - 1j * py / sqrtp)
        cc = sign * (px / sqrtp + 1j * py / sqrtp)
        dd = sign * pz / sqrtp
        E = [[0.5 + aa, 0., dd, bb], [0., 0.5 + aa, cc, -dd], [dd, bb, 0.5 - aa, 0.], [cc, -dd, 0., 0.5 - aa]]
        f = [np.fft.fftn(p) for p in self.Psi_init]
        out = [sum(E[i][j] * f[j] for j in range(4)) for i in range(4)]
        self.Psi1_init, self.Psi2_init, self.Psi3_init, self.Psi4_init = [np.fft.ifftn(o) for o in out]
        self.Psi_init = np.array([self.Psi1_init, self.Psi2_init, self.Psi3_init, self.Psi4_init])

    def Density_From_Spinor(self, Psi):
        return sum(np.abs(Psi[k]) ** 2 for k in range(4))

    def Norm(self, Psi):
        norm = sum(np.sum(np.abs(Psi[k]) ** 2) for k in range(4))
        return np.sqrt(norm * self.dX * self.dY * self.dZ)

    # ------------------------------------------------------------------ run
    def propagate(self, psi, n_steps, t_index0=0, continue_run=False, stream=None):
        """Advance the device spinor ``psi`` (torch complex128 (4, Z, Y, X), in place)
        by ``n_steps`` propagations at t = dt*(t_index0 + k), k = 1..n_steps; without
        ``continue_run`` it is normalised first.  Returns the (n_steps, 12) samples
        (x, y, z, alpha1, alpha2, alpha3, A0, px, py, pz, K, norm)."""
        torch = _torch()
        if psi.dtype != torch.complex128 or not psi.is_cuda or not psi.is_contiguous() or \
                tuple(psi.shape) != (4, self.Z_gridDIM, self.Y_gridDIM, self.X_gridDIM):
            raise _lib.WignerArgumentError('psi must be a contiguous CUDA complex128 tensor (4, Z, Y, X)')
        obs = np.empty((n_steps, _lib.DIRAC3_NOBS))
        st = stream if stream is not None else torch.cuda.current_stream(psi.device)
        flags = _lib.WIG_RUN_CONTINUE if continue_run else 0
        check(_lib.load().dirac3_run(self._handle, psi.data_ptr(), t_index0, n_steps, flags, dptr(obs),
                                     st.cuda_stream), 'dirac3_run')
        return obs

    def Run(self):
        torch = _torch()
        P0 = np.ascontiguousarray(np.asarray(self.Psi_init), dtype=np.complex128)
        if P0.shape != (4, self.Z_gridDIM, self.Y_gridDIM, self.X_gridDIM):
            raise _lib.WignerArgumentError('Psi_init must have shape (4, Z_gridDIM, Y_gridDIM, X_gridDIM)')
        self.Psi1_init, self.Psi2_init, self.Psi3_init, self.Psi4_init = P0
        dev = torch.device('cuda', self._device)
        n = int(self.timeSteps)
        skip = max(int(self.skipFrames), 1)
        fileName = getattr(self, 'fileName', '')
        sink = None
        if fileName:                                       # :1267-1293
            sink = frames.open_write(fileName)
            frames.dirac3_header(sink, self)
        emit = frames.dirac3_frame(self.frameSaveMode, sink is not None)
        self.frames = {0: frames.copy_frame(emit(sink, 0, P0))}   # the initial spinor (:1310-1315)
        obs = np.empty((n, _lib.DIRAC3_NOBS))
        with torch.cuda.device(dev):
            psi = torch.from_numpy(P0.copy()).to(dev)
            writer = frames.FrameWriter(psi, sink, emit, keep=self.frames)
            try:
                t = 0
                while t < n:
                    nxt = min(n, (t // skip + 1) * skip)
                    obs[t:nxt] = self.propagate(psi, nxt - t, t_index0=t, continue_run=t > 0)
                    t = nxt
                    if t % skip == 0:                      # after step t (:1454-1461)
                        writer.capture(t, psi)
                self.Psi_end = psi.cpu().numpy()
            finally:
                writer.close()
        if sink is not None:
            sink.close()
        self.Psi_init = P0
        self.timeRange = np.arange(1, n + 1)
        (self.X_average, self.Y_average, self.Z_average, self.Alpha1_average, self.Alpha2_average,
         self.Alpha3_average, self.Potential_0_average) = [obs[:, k].copy() for k in range(7)]
        if getattr(self, 'Compute_Ehrenfest_P', True):
            (self.Px_average, self.Py_average, self.Pz_average,
             self.K_Energy_average) = [obs[:, k].copy() for k in range(7, 11)]
        else:
            self.Px_average = self.Py_average = self.Pz_average = self.K_Energy_average = np.zeros(0)
        self.Norm_average = obs[:, 11].copy()
        return 0

    def load_Density(self, n, fileName=None):
        """The density frame of step ``n`` (``load_Density`` :1096-1106)."""
        return frames.read(fileName or self.fileName, '/' + str(n))

    def load_Spinor(self, n, fileName=None):
        """The two slices ``save_Spinor_SliceYZ`` wrote at step ``n``: (xy at z index
        0, xz at y index 0), each (4, ., X).  The reference's ``load_Spinor``
        (:1108-1123) reads keys its Run does not write."""
        f = frames.open_read(fileName or self.fileName)
        try:
            out = []
            for plane in ('xy', 'xz'):
                out.append(np.array([np.array(f['%s/%d/real/%d' % (plane, k, n)][...]) +
                                     1j * np.array(f['%s/%d/imag/%d' % (plane, k, n)][...]) for k in range(1, 5)]))
            return tuple(out)
        finally:
            f.close()
