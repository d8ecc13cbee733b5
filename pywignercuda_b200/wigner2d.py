"""Drop-in Wigner2D propagators: ``GPU_Wigner2D_FFT`` and ``GPU_Wigner2D_ODM2``.

Same construction protocol as the reference (``GPU_Wigner2D_FFT.py:529-1964``):
an instance subclass sets ``dampingFunction``, ``grossPitaevskiiCoefficient``,
``fp_Damping_String`` (and ``epsilon`` / ``L_material`` for ODM), calls
``SetTimeTrack(dt, timeSteps, skipFrames, fileName)`` and then the class
constructor with the grid, amplitudes, hbar, mass, diffusion, damping and the
potential / derivative / kinetic expression strings; it sets ``W_init`` (FFT-
shifted (P_gridDIM, X_gridDIM) array) and calls ``Run()``.  ``Run()`` returns 0
and leaves ``timeRange``, ``X_average``, ``X2_average``, ``P_average``,
``P2_average``, ``XP_average``, ``dPotentialdX_average``,
``PdPotentialdX_average``, ``XdPotentialdX_average``, ``Hamiltonian_average``,
``negativeArea`` and ``W_end`` on the instance (``:1918-1954``), plus
``Norm_average`` (dX dP sum W of each sample) and ``frames`` (the W saved every
``skipFrames`` steps, ``save_Frame`` :660-663).  With ``fileName`` set, the run
writes the reference's file layout (``frames.py``): HDF5 when h5py is
importable, else ``fileName + '.npz'`` with the same keys.

The propagation runs on the GPU through ``libwigner_b200.so``; device memory
and the stream come from PyTorch.  There is no CPU path.
"""
import ctypes

import numpy as np

from . import _lib, frames
from ._lib import WigDesc, check, dptr


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise _lib.WignerCudaError('no CUDA device: the propagators run on the GPU only')
    return torch


def _eval(expr, **variables):
    """The reference's host-side evaluation of expression strings
    (``eval(s, np.__dict__, locals())`` with ``pow = np.power``, :674-692)."""
    ns = dict(np.__dict__)
    ns.update(pow=np.power, atan=np.arctan, M_E=np.e, sqrt=np.sqrt, exp=np.exp, fabs=np.fabs)
    ns.update(variables)
    return eval(expr, ns)


class Propagator_Base:
    """Grid, helpers and initial states of the reference's ``Propagator_Base``
    (``GPU_Wigner2D_FFT.py:529-1705``) that instances use on the host."""

    constants_mode = _lib.CONST_CUDA_F     # '%f' kernel constants, as the reference

    def SetTimeTrack(self, dt, timeSteps=128, skipFrames=1, fileName='', compression=None):
        self.runTime = float(dt) * timeSteps
        self.timeSteps = timeSteps
        self.dt = dt
        self.skipFrames = skipFrames
        self.fileName = fileName
        self.compression = compression

    def SetPhaseSpaceBox2D(self, X_gridDIM, P_gridDIM, X_amplitude, P_amplitude):
        self.X_gridDIM = X_gridDIM
        self.P_gridDIM = P_gridDIM
        self.X_amplitude = X_amplitude
        self.P_amplitude = P_amplitude
        self.dX = 2. * X_amplitude / float(X_gridDIM)
        self.dP = 2. * P_amplitude / float(P_gridDIM)
        self.dTheta = 2. * np.pi / (2. * P_amplitude)
        self.Theta_amplitude = self.dTheta * P_gridDIM / 2.
        self.dLambda = 2. * np.pi / (2. * X_amplitude)
        self.Lambda_amplitude = self.dLambda * X_gridDIM / 2.
        self.SetPhaseSpaceGrid2D()

    def SetPhaseSpaceGrid2D(self):
        self.X_range = np.linspace(-self.X_amplitude, self.X_amplitude - self.dX, self.X_gridDIM)
        self.Lambda_range = np.linspace(-self.Lambda_amplitude, self.Lambda_amplitude - self.dLambda,
                                        self.X_gridDIM)
        self.Theta_range = np.linspace(-self.Theta_amplitude, self.Theta_amplitude - self.dTheta,
                                       self.P_gridDIM)
        self.P_range = np.linspace(-self.P_amplitude, self.P_amplitude - self.dP, self.P_gridDIM)
        self.X = np.fft.fftshift(self.X_range)[np.newaxis, :]
        self.Theta = np.fft.fftshift(self.Theta_range)[:, np.newaxis]
        self.Lambda = np.fft.fftshift(self.Lambda_range)[np.newaxis, :]
        self.P = np.fft.fftshift(self.P_range)[:, np.newaxis]

    # ---- expression strings evaluated on the host (:674-692, :1674-1681); the
    # strings may use cf[0..7], the instance's optional ``coefficients``
    def _coef(self):
        c = np.zeros(8)
        coefs = getattr(self, 'coefficients', None)
        if coefs is not None:
            c[:len(coefs)] = coefs
        return c

    def Potential(self, t, x):
        return _eval(self.potentialString, t=t, x=x, cf=self._coef())

    def dPotential(self, t, x):
        return _eval(self.dPotentialString, t=t, x=x, cf=self._coef())

    def fp_Damping(self, p):
        return _eval(self.fp_Damping_String, p=p, cf=self._coef())

    # ---- helpers
    def fft_shift2D(self, X):
        return np.fft.fftshift(np.fft.fftshift(X, axes=1), axes=0)

    def WignerMarginal_Probability_x(self, W):
        return np.sum(W, axis=0) * self.dP

    def WignerMarginal_Probability_p(self, W):
        return np.sum(W, axis=1) * self.dX

    def Fourier_Theta_To_P_CPU(self, W):
        return np.fft.ifft(W, axis=0)

    def Fourier_P_To_Theta_CPU(self, W):
        return np.fft.fft(W, axis=0)

    def Fourier_X_To_Lambda_CPU(self, W):
        return np.fft.fft(W, axis=1)

    def Fourier_Lambda_To_X_CPU(self, W):
        return np.fft.ifft(W, axis=1)

    # ---- initial states (:715-771)
    def Wigner_HarmonicOscillator(self, n, omega, x, p):
        from scipy.special import eval_laguerre
        self.representation = 'x_p'
        r2 = self.mass * omega ** 2 * ((self.X - x)) ** 2 + ((self.P - p)) ** 2 / self.mass
        W = (-1) ** (n) * eval_laguerre(n, 2 * r2) * np.exp(-r2)
        norm = np.sum(W) * self.dX * self.dP
        return W / norm

    def Heaviside(self, x):
        return 0.5 * (np.sign(x) + 1.)

    def Psi_Half_HarmonicOscillator(self, n, omega, x0, p0, X):
        from scipy.special import eval_legendre
        k = np.sqrt(self.mass * omega / self.hBar)
        return (np.exp(1j * p0) * np.exp(-0.5 * k ** 2 * (X - x0) ** 2) * eval_legendre(n, k * (X - x0))
                * self.Heaviside(-(X - x0)))

    def Wigner_Half_HarmonicOscillator(self, n, omega, x0, p0):
        X_minus = self.X_range[np.newaxis, :] - 0.5 * self.hBar * self.Theta_range[:, np.newaxis]
        X_plus = self.X_range[np.newaxis, :] + 0.5 * self.hBar * self.Theta_range[:, np.newaxis]
        W = (self.Psi_Half_HarmonicOscillator(n, omega, x0, p0, X_minus)
             * self.Psi_Half_HarmonicOscillator(n, omega, x0, p0, X_plus).conj())
        W = self.Fourier_Theta_To_P_CPU(np.fft.fftshift(W))
        return W / (np.sum(W) * self.dX * self.dP)

    def Wigner_FromWavefunction(self, psi):
        """Wigner function of a wave-function callable psi(x), by the same discrete
        transform as ``Wigner_Half_HarmonicOscillator`` (psi(x - hbar theta/2)
        psi*(x + hbar theta/2), IFFT over theta), shifted layout, normalised.
        This package's helper: the reference has no counterpart (its classes take
        W_init as an array)."""
        X_minus = self.X_range[np.newaxis, :] - 0.5 * self.hBar * self.Theta_range[:, np.newaxis]
        X_plus = self.X_range[np.newaxis, :] + 0.5 * self.hBar * self.Theta_range[:, np.newaxis]
        W = psi(X_minus) * np.conj(psi(X_plus))
        W = self.Fourier_Theta_To_P_CPU(np.fft.fftshift(W))
        return W / (np.sum(W) * self.dX * self.dP)

    # ---- classical reference trajectories (:597-657)
    def symplecticExpK(self, mass, dt, c, Z):
        return Z + np.array([dt * c * Z[1] / mass, 0])

    def symplecticExpV(self, mass, dt, d, dVdx, Z):
        return Z + np.array([0, -dt * d * dVdx(0., Z[0])])

    def symplecticExpKExpV2(self, mass, dt, dVdx, Z0):
        Z = self.symplecticExpK(mass, dt, 0.5, self.symplecticExpV(mass, dt, 1.0, dVdx, Z0))
        return self.symplecticExpK(mass, dt, 0.5, self.symplecticExpV(mass, dt, 0.0, dVdx, Z))

    def SymplecticPropagator(self, dt, n_iterations, Z0, gammaDamping):
        Z = np.asarray(Z0, dtype=float)
        trajectory = []
        for i in range(n_iterations):
            trajectory.append(np.append(Z, dt * (i + 1)))
            Z = self.symplecticExpKExpV2(self.mass, dt, self.dPotential, Z)
            Z[1] = np.exp(-2. * gammaDamping * dt) * Z[1]
        return np.array(trajectory)


class GPU_Wigner2D_FFT(Propagator_Base):
    """Wigner propagator with diffusion and Caldeira-Leggett / ODM damping
    (``GPU_Wigner2D_FFT.py:1713-1964``)."""

    _odm2 = False
    _kvn = False
    _strang_gp = False

    def __init__(self, X_gridDIM, P_gridDIM, X_amplitude, P_amplitude, hBar, mass, D_Theta, D_Lambda,
                 gammaDamping, potentialString, dPotentialString, kinematicString, normalization='Wigner'):
        self.normalization = normalization
        self.D_Theta = D_Theta
        self.D_Lambda = D_Lambda
        self.gammaDamping = gammaDamping
        self.potentialString = potentialString
        self.dPotentialString = dPotentialString
        self.kinematicString = kinematicString
        self.SetPhaseSpaceBox2D(X_gridDIM, P_gridDIM, X_amplitude, P_amplitude)
        self.hBar = hBar
        self.mass = mass
        self._build()

    def _damping_code(self):
        kind = getattr(self, 'dampingFunction', 'CaldeiraLeggett')
        if kind == 'CaldeiraLeggett':
            return _lib.DAMP_CALDEIRA_LEGGETT
        if kind == 'ODM':
            return _lib.DAMP_ODM
        return _lib.DAMP_NONE

    def _build(self):
        if not self._strang_gp and getattr(self, 'grossPitaevskiiCoefficient', 0.) != 0.:
            raise _lib.WignerUnsupportedError('the Gross-Pitaevskii term is not part of this propagator')
        if not hasattr(self, 'fp_Damping_String'):
            self.fp_Damping_String = 'fabs(p)'
        for name in ('dt', 'timeSteps'):
            if not hasattr(self, name):
                raise _lib.WignerArgumentError('call SetTimeTrack(dt, timeSteps, ...) before the constructor')
        lib = _lib.load()
        # host tables of Run (:1747, :1785-1792), evaluated with numpy like the reference
        self._x_tab = np.ascontiguousarray(self.X[0], dtype=np.float64)
        self._p_tab = np.ascontiguousarray(self.P[:, 0], dtype=np.float64)
        self._theta_tab = np.ascontiguousarray(self.Theta[:, 0], dtype=np.float64)
        self._lambda_tab = np.ascontiguousarray(self.Lambda[0], dtype=np.float64)
        self._dv_tab = np.ascontiguousarray(
            np.broadcast_to(self.dPotential(0., self.X), self.X.shape)[0], dtype=np.float64)
        self._v0_tab = np.ascontiguousarray(
            np.broadcast_to(self.Potential(0, self.X), self.X.shape)[0], dtype=np.float64)
        self.Hamiltonian = self.fft_shift2D(self.P ** 2 / (2. * self.mass) + self.Potential(0, self.X))
        d = WigDesc()
        d.abi_version = _lib.ABI_VERSION
        d.n_x, d.n_p = int(self.X_gridDIM), int(self.P_gridDIM)
        d.damping = self._damping_code()
        d.kinetic_from_string = 1 if (self._odm2 or self._strang_gp) else 0
        d.constants = self.constants_mode
        d.precision = _lib.PREC_C128
        d.n_lindblad = 2 if self._odm2 else 1
        d.potential_phase = _lib.PHASE_KVN if self._kvn else _lib.PHASE_MOYAL
        d.skip_normalise = 1 if (self._kvn and self.normalization != 'Wigner') else 0
        d.splitting = _lib.SPLIT_STRANG_GP if self._strang_gp else _lib.SPLIT_LIE
        d.gp_coefficient = float(getattr(self, 'GPitaevskiiCoeff', 0.)) if self._strang_gp else 0.
        d.x_amplitude, d.p_amplitude = float(self.X_amplitude), float(self.P_amplitude)
        d.hbar, d.mass, d.dt = float(self.hBar), float(self.mass), float(self.dt)
        d.d_theta, d.d_lambda, d.gamma = float(self.D_Theta), float(self.D_Lambda), float(self.gammaDamping)
        d.epsilon = float(getattr(self, 'epsilon', 0.5))
        d.l_material = float(getattr(self, 'L_material', 1.0))
        d.weight1 = float(getattr(self, 'weightLindbland1', 1.0))
        d.weight2 = float(getattr(self, 'weightLindbland2', 0.0))
        self._strings = [s.encode() for s in (self.potentialString, self.kinematicString,
                                              self.fp_Damping_String, self.dPotentialString)]
        d.potential, d.kinetic, d.fp_damping, d.dpotential = self._strings
        d.x_table, d.p_table = dptr(self._x_tab), dptr(self._p_tab)
        d.theta_table, d.lambda_table = dptr(self._theta_tab), dptr(self._lambda_tab)
        d.dv_table, d.v0_table = dptr(self._dv_tab), dptr(self._v0_tab)
        for i, v in enumerate(self._coef()):
            d.coef[i] = float(v)
        self._desc = d
        torch = _torch()
        self._device = torch.cuda.current_device()
        h = ctypes.c_void_p()
        check(lib.wig_create(d, h), 'wig_create')
        self._handle = h

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                _lib.load().wig_destroy(h)
            except Exception:
                pass
            h.value = None

    # ------------------------------------------------------------------ run
    def propagate(self, W, n_prop, t_index0=0, continue_run=False, stream=None):
        """Advance the device array ``W`` (torch complex128 (P, X), in place) by
        ``n_prop`` propagations; returns the (n_prop+1, 11) observables
        (norm, x, x^2, p, p^2, xp, V', pV', xV', H, negative area)."""
        torch = _torch()
        if W.dtype != torch.complex128 or not W.is_cuda or not W.is_contiguous() or \
                tuple(W.shape) != (self.P_gridDIM, self.X_gridDIM):
            raise _lib.WignerArgumentError('W must be a contiguous CUDA complex128 tensor of shape (P, X)')
        obs = np.empty((n_prop + 1, _lib.WIG_NOBS))
        st = stream if stream is not None else torch.cuda.current_stream(W.device)
        flags = _lib.WIG_RUN_CONTINUE if continue_run else 0
        check(_lib.load().wig_run(self._handle, W.data_ptr(), t_index0, n_prop, flags, dptr(obs),
                                  st.cuda_stream), 'wig_run')
        return obs

    def _frame_writer(self, W):
        """The output file (when ``fileName`` is set) with its header, and the
        asynchronous frame writer that fills ``frames`` and the file."""
        sink = None
        if self.fileName:
            sink = frames.open_write(self.fileName)
            frames.wigner_header(sink, self)
        self.frames = {}
        emit = frames.wigner_frame if sink is not None else (lambda f, key, W: W)
        return sink, frames.FrameWriter(W, sink, emit, keep=self.frames)

    def WignerFunctionFromFile(self, n, fileName=None):
        """The frame saved at step ``n`` (``WignerFunctionFromFile`` :908-917)."""
        return frames.read(fileName or self.fileName, '/' + str(n))

    def LoadEhrenfestFromFile(self):
        """The observables and the first / last states of a run's file (:919-940)."""
        frames.load_ehrenfest(self, self.fileName)

    def Run(self):
        torch = _torch()
        W0 = np.ascontiguousarray(self.W_init, dtype=np.complex128)
        if W0.shape != (self.P_gridDIM, self.X_gridDIM):
            raise _lib.WignerArgumentError('W_init must have shape (P_gridDIM, X_gridDIM)')
        dev = torch.device('cuda', self._device)
        with torch.cuda.device(dev):
            W = torch.from_numpy(W0.copy()).to(dev)
            n_total = int(self.timeSteps) + 1             # Run :1776 loops over 0..timeSteps
            skip = max(int(self.skipFrames), 1)
            obs = np.empty((n_total + 1, _lib.WIG_NOBS))
            sink, writer = self._frame_writer(W)
            saved = []
            t, cont = 0, False
            try:
                while t < n_total:
                    if t % skip == 0 and t <= self.timeSteps:
                        if not cont:                       # W must be normalised first
                            obs[0] = self.propagate(W, 0)[0]
                            cont = True
                        writer.capture(t, W)               # the sample before step t (:1880-1882)
                        saved.append(t)
                    nxt = min(n_total, (t // skip + 1) * skip)
                    o = self.propagate(W, nxt - t, t_index0=t, continue_run=cont)
                    obs[t:nxt + 1] = o
                    t, cont = nxt, True
                W_end = W.cpu().numpy()
            finally:
                writer.close()
        n = int(self.timeSteps) + 1
        self.timeRange = np.arange(n) * self.dt
        self.timeRangeIndexSaved = saved
        self.Norm_average = obs[:n, 0].copy()
        (self.X_average, self.X2_average, self.P_average, self.P2_average, self.XP_average,
         self.dPotentialdX_average, self.PdPotentialdX_average, self.XdPotentialdX_average,
         self.Hamiltonian_average, self.negativeArea) = [obs[:n, k].copy() for k in range(1, 11)]
        self.W_end_complex = W_end
        self.W_end = W_end.real.copy()
        if sink is not None:
            frames.wigner_tail(sink, self)
            sink.close()
        return 0


class GPU_Wigner2D_ODM2(GPU_Wigner2D_FFT):
    """Kinetic phase from the kinetic string and two Lindblad terms, one damping
    and one pumping (``GPU_Wigner2D_FFT.py:1973-2230``)."""

    _odm2 = True

    def __init__(self, X_gridDIM, P_gridDIM, X_amplitude, P_amplitude, hBar, mass, D_Theta, D_Lambda,
                 gammaDamping, weightLindbland1, weightLindbland2, potentialString, dPotentialString,
                 kinematicString, normalization='Wigner'):
        self.weightLindbland1 = weightLindbland1
        self.weightLindbland2 = weightLindbland2
        GPU_Wigner2D_FFT.__init__(self, X_gridDIM, P_gridDIM, X_amplitude, P_amplitude, hBar, mass,
                                  D_Theta, D_Lambda, gammaDamping, potentialString, dPotentialString,
                                  kinematicString, normalization)


class GPU_FokkerPlank2D_FFT(GPU_Wigner2D_FFT):
    """Classical (Koopman-von Neumann / Liouville) propagator in phase space
    with diffusion and Caldeira-Leggett damping (``GPU_Wigner2D_FFT.py:2242-2459``):
    the Wigner step with the Moyal potential factor replaced by
    exp(+i dt V'(t, x) theta), V' from ``dPotentialString``
    (``exp_PotentialKvN_source`` :27-75); damped steps renormalise only when
    ``normalization == 'Wigner'`` (:2404-2406).  The kinetic pass is the Wigner
    one (p lambda / m); an instance may set ``kinematicString`` first, as the
    reference's compile step expects it."""

    _kvn = True

    def __init__(self, X_gridDIM, P_gridDIM, X_amplitude, P_amplitude, hBar, mass, D_Theta, D_Lambda,
                 gammaDamping, potentialString, dPotentialString, normalization='Wigner'):
        GPU_Wigner2D_FFT.__init__(self, X_gridDIM, P_gridDIM, X_amplitude, P_amplitude, hBar, mass,
                                  D_Theta, D_Lambda, gammaDamping, potentialString, dPotentialString,
                                  getattr(self, 'kinematicString', '0.5*p*p'), normalization)


class GPU_Wigner2D_GPitaevskii(GPU_Wigner2D_FFT):
    """Wigner propagator with the Strang splitting and the Gross-Pitaevskii
    term of ``GPU_Wigner2D_GPitaevskii.py:1767-2060``: per step, half potential
    (with the mean-field phase from the x-marginal when ``GPitaevskiiCoeff``
    != 0), kinetic (from ``kinematicString``), half potential, damping
    (Caldeira-Leggett or ODM) and, if damped, normalisation.  An instance sets
    ``GPitaevskiiCoeff`` (and ``dampingFunction``, ``fp_Damping_String``, ...)
    before calling the constructor.  ``Run()`` records the observables after
    every step (``timeSteps + 1`` steps) and, with the mean-field term,
    ``ProbabilitySquare_average`` = sum_x P(x)^2 dx after each kinetic step."""

    _strang_gp = True

    def __init__(self, X_gridDIM, P_gridDIM, X_amplitude, P_amplitude, hBar, mass, D_Theta, D_Lambda,
                 gammaDamping, potentialString, dPotentialString, kinematicString, normalization='Wigner'):
        if not hasattr(self, 'GPitaevskiiCoeff'):
            self.GPitaevskiiCoeff = 0.
        GPU_Wigner2D_FFT.__init__(self, X_gridDIM, P_gridDIM, X_amplitude, P_amplitude, hBar, mass,
                                  D_Theta, D_Lambda, gammaDamping, potentialString, dPotentialString,
                                  kinematicString, normalization)

    def probability_square(self, n):
        """sum_x P(x)^2 dx after each of the last ``propagate`` call's first n steps."""
        out = np.empty(n)
        check(_lib.load().wig_run_probability_square(self._handle, dptr(out), n), 'wig_run_probability_square')
        return out

    def Run(self):
        torch = _torch()
        W0 = np.ascontiguousarray(self.W_init, dtype=np.complex128)
        if W0.shape != (self.P_gridDIM, self.X_gridDIM):
            raise _lib.WignerArgumentError('W_init must have shape (P_gridDIM, X_gridDIM)')
        n = int(self.timeSteps) + 1                        # Run :1897 loops over 0..timeSteps
        skip = max(int(self.skipFrames), 1)
        dev = torch.device('cuda', self._device)
        after = np.empty((n, _lib.WIG_NOBS))
        psq = []
        saved = []
        with torch.cuda.device(dev):
            W = torch.from_numpy(W0.copy()).to(dev)
            sink, writer = self._frame_writer(W)
            try:
                t = 0                                      # steps done
                while t < n:
                    # frames follow step tIndex for tIndex % skipFrames == 0 (:1996-1999)
                    nxt = 1 if t == 0 else ((t - 1) // skip + 1) * skip + 1
                    end = min(nxt, n)
                    o = self.propagate(W, end - t, t_index0=t, continue_run=t > 0)
                    after[t:end] = o[1:]                   # row k + 1: after step k of the chunk
                    if self.GPitaevskiiCoeff != 0.:
                        psq.append(self.probability_square(end - t))
                    if end == nxt:
                        writer.capture(nxt - 1, W)
                        saved.append(nxt - 1)
                    t = end
                W_end = W.cpu().numpy()
            finally:
                writer.close()
        self.timeRange = np.arange(n) * self.dt
        self.timeRangeIndexSaved = saved
        self.Norm_average = after[:, 0].copy()
        (self.X_average, self.X2_average, self.P_average, self.P2_average, self.XP_average,
         self.dPotentialdX_average, self.PdPotentialdX_average, self.XdPotentialdX_average,
         self.Hamiltonian_average, self.negativeArea) = [after[:, k].copy() for k in range(1, 11)]
        self.ProbabilitySquare_average = np.concatenate(psq) if psq else np.zeros(0)
        self.W_end_complex = W_end
        self.W_end = W_end.real.copy()
        if sink is not None:
            frames.wigner_tail(sink, self, extra=(('ProbabilitySquare_average', 'ProbabilitySquare_average'),))
            sink.close()
        return 0


class GPU_Wigner2D_GPitaevskii_Bloch(GPU_Wigner2D_GPitaevskii):
    """Imaginary-time (Bloch) propagator of ``GPU_Wigner2D_GPitaevskii.py:2064-2545``
    for ground states (``Run``) and the first excited state (``Run_ExitedState1``):
    Strang steps with real exponentials and the mean-field term (set
    ``GPitaevskiiCoeff`` before the constructor), normalisation every step, and
    the reference's step control -- a step counts only if the total energy
    (Hamiltonian K(P) + V(0, X) plus the mean-field energy) falls and
    |purity| < 1 (and, for the excited state, no p-marginal value is negative);
    otherwise the step size is halved and the last counted state restored.
    Deviations: ``GPitaevskiiCoeff = 0`` works (the reference's ``Run`` reads its
    marginal buffer before creating it, :2145-2176); the excited-state check
    uses the p-marginal itself (the reference's ``ProbabilityP`` indexes rows
    with the row stride and writes past its output, :432-441, :1750-1755)."""

    def __init__(self, X_gridDIM, P_gridDIM, X_amplitude, P_amplitude, hBar, mass, potentialString,
                 kinematicString):
        self.dampingFunction = 'CaldeiraLeggett'
        self.fp_Damping_String = '0.'
        GPU_Wigner2D_GPitaevskii.__init__(self, X_gridDIM, P_gridDIM, X_amplitude, P_amplitude, hBar, mass,
                                          0., 0., 0., potentialString, '0.', kinematicString)
        # the Bloch class's Hamiltonian uses the kinetic string (:2097-2101)
        self.Hamiltonian = self.fft_shift2D(self.KineticEnergy(self.P) + self.Potential(0, self.X) + 0. * self.P)

    def KineticEnergy(self, p):
        return _eval(self.kinematicString, p=p, cf=self._coef())

    def _stats(self, W, normalise):
        out = np.empty(_lib.WIG_BLOCH_NSTATS)
        st = _torch().cuda.current_stream(W.device)
        check(_lib.load().wig_bloch_stats(self._handle, W.data_ptr(), int(normalise), dptr(out), st.cuda_stream),
              'wig_bloch_stats')
        return out

    def _step(self, W, t_index, dtb, W0=None):
        out = np.empty(_lib.WIG_BLOCH_NSTATS)
        st = _torch().cuda.current_stream(W.device)
        check(_lib.load().wig_bloch_step(self._handle, W.data_ptr(), int(t_index), float(dtb),
                                         W0.data_ptr() if W0 is not None else None, dptr(out), st.cuda_stream),
              'wig_bloch_step')
        return out

    def _relax(self, W0_ground, time_steps):
        torch = _torch()
        init = np.ascontiguousarray(self.W_init, dtype=np.complex128)
        if init.shape != (self.P_gridDIM, self.X_gridDIM):
            raise _lib.WignerArgumentError('W_init must have shape (P_gridDIM, X_gridDIM)')
        dev = torch.device('cuda', self._device)
        with torch.cuda.device(dev):
            W = torch.from_numpy(init.copy()).to(dev)
            W_step = torch.from_numpy(init.copy()).to(dev)      # the reference keeps W_init here (:2135)
            s0 = self._stats(W, True)
            energy = s0[4] + s0[7]
            dtb = float(self.dt)
            avg, hist_e, hist_nle, hist_pur = [], [], [], []
            for t_index in range(time_steps + 1):
                s = self._step(W, t_index, dtb, W0_ground)
                avg.append(s[:5].copy())
                e_step = s[4] + s[7]
                purity = complex(s[5], s[6])
                if t_index > 0:
                    if e_step < energy and abs(purity) < 1. and s[8] == 0.:
                        W_step.copy_(W)
                        hist_pur.append(purity.real)
                        hist_e.append(e_step)
                        energy = e_step
                        hist_nle.append(s[7])
                    else:
                        dtb = dtb / 2.
                        W.copy_(W_step)
            torch.cuda.synchronize(dev)
            W_end = W.cpu().numpy()
        avg = np.array(avg)
        self.timeRange = np.arange(time_steps + 1) * self.dt
        (self.X_average, self.X2_average, self.P_average, self.P2_average,
         self.Hamiltonian_average) = [avg[:, k].copy() for k in range(5)]
        self.TotalEnergyHistory = np.array(hist_e)
        if self.GPitaevskiiCoeff != 0.:
            self.NonLinearEnergyHistory = np.array(hist_nle)
        self.purity = np.array(hist_pur)
        return W_end

    def Run(self):
        W_end = self._relax(None, int(self.timeSteps))
        self.W_0_complex = W_end
        self.W_0 = W_end.real.copy()
        if self.fileName:                                  # :2112-2115, :2300-2330
            f = frames.open_write(self.fileName)
            frames.wigner_header(f, self)
            f['timeRange'] = self.timeRange
            f['timeRangeIndexSaved'] = np.zeros(0, dtype=np.int64)
            for key, attr in (('X_Ehrenfest', 'X_average'), ('X2_Ehrenfest', 'X2_average'),
                              ('P_Ehrenfest', 'P_average'), ('P2_Ehrenfest', 'P2_average'),
                              ('Hamiltonian_average', 'Hamiltonian_average')):
                f['/Ehrenfest/' + key] = getattr(self, attr)
            f['/Potential'] = np.broadcast_to(self.Potential(0, self.X_range), self.X_range.shape)
            f['/PotentialString'] = self.potentialString
            f['W_init'] = np.real(np.asarray(self.W_init))
            f['W_0'] = self.W_0
            f.close()
        return 0

    def Run_ExitedState1(self, timeSteps=None):
        if not hasattr(self, 'W_0_complex'):
            raise _lib.WignerArgumentError('Run() must find the ground state W_0 first')
        torch = _torch()
        W0 = torch.from_numpy(np.ascontiguousarray(self.W_0_complex)).to(torch.device('cuda', self._device))
        W_end = self._relax(W0, int(self.timeSteps if timeSteps is None else timeSteps))
        self.W_1 = W_end.real.copy()
        if self.fileName:                                  # :2532 adds W_1 to Run's file
            frames.append(self.fileName, 'W_1', self.W_1)
        return 0
