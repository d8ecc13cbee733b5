"""CPU oracle: the reference notebook's own CPU propagator (TEST INFRASTRUCTURE).

Restates ``CPU_GPU_Wigner2D.ipynb`` cells ``SetGrid`` / ``SetExponentials`` /
``Propagation_Step`` / ``Run`` / ``InitialState`` (raw-JSON lines 93-290,
360-496): real W (float64), unshifted x/p grids, ``fftfreq`` theta/lambda
half-grids (the Nyquist entry is negative), a Strang step V/2 - K - V/2 with
real FFTs and normalised inverses, hbar = 1 hard-wired.  pyFFTW (absent here)
is replaced by ``scipy.fft.rfft/irfft`` with the same conventions (forward
unnormalised, backward normalised, the imaginary part of the DC and Nyquist
bins ignored on the way back).

Known answer recorded in the notebook (``CPU_GPU_Wigner2D.ipynb:557,577``):
512x512, amplitudes 12, dt = 0.05, V = 0.5x^2 + 0.01x^4, K = p^2/2,
W0 ~ exp(-((p-3)^2 + x^2)), 500 steps:
    min W              = -0.16857913679981978
    sum W dx dp        =  1.0000000000000249
"""
import numpy as np
import scipy.fft as sfft

from .common import WORKERS, eval_expr

KNOWN_MIN_W = -0.16857913679981978
KNOWN_NORM = 1.0000000000000249


class StrangNotebook:
    def __init__(self, n_x=512, n_p=512, x_amplitude=12., p_amplitude=12., dt=0.05,
                 potential=' 0.5*pow(X,2) + 0.01*pow(X,4) ', kinetic=' pow(P,2)/(2.)'):
        self.n_x, self.n_p, self.dt = n_x, n_p, dt
        # SetGrid (notebook cell 6)
        dX = 2. * x_amplitude / n_x
        dP = 2. * p_amplitude / n_p
        X = np.linspace(-x_amplitude, x_amplitude - dX, n_x)[np.newaxis, :]
        Lam = np.fft.fftfreq(n_x, dX / (2 * np.pi))[:(1 + n_x // 2)][np.newaxis, :]
        P = np.linspace(-p_amplitude, p_amplitude - dP, n_p)[:, np.newaxis]
        Th = np.fft.fftfreq(n_p, dP / (2 * np.pi))[:(1 + n_p // 2)][:, np.newaxis]
        self.X, self.P, self.Theta, self.Lambda = X, P, Th, Lam
        self.dX, self.dP = 2. * x_amplitude / float(n_x), 2. * p_amplitude / float(n_p)

        def V(x):
            return eval_expr(potential, X=x)

        def K(p):
            return eval_expr(kinetic, P=p)
        # SetExponentials (cell 7)
        self.expV = np.exp(-dt * 0.5j * (V(X - 0.5 * Th) - V(X + 0.5 * Th)))
        self.expK = np.exp(-dt * 1j * (K(P + 0.5 * Lam) - K(P - 0.5 * Lam)))

    def initial_state(self):
        """``InitialState`` (cell 21): exp(-((P-3)^2/m + m w^2 X^2)), normalised."""
        mass, omega = 1., 1.
        W = np.exp(-((self.P - 3) ** 2 / mass + mass * omega ** 2 * (self.X) ** 2))
        W = W + 0. * self.X * self.P
        norm = np.sum(W) * self.dX * self.dP
        return W / norm

    def step(self, W):
        """``Propagation_Step`` (cell 10): V/2, K, V/2 with real FFTs."""
        B = sfft.rfft(W, axis=0, workers=WORKERS)
        B *= self.expV
        W = sfft.irfft(B, n=self.n_p, axis=0, workers=WORKERS)
        Z = sfft.rfft(W, axis=1, workers=WORKERS)
        Z *= self.expK
        W = sfft.irfft(Z, n=self.n_x, axis=1, workers=WORKERS)
        B = sfft.rfft(W, axis=0, workers=WORKERS)
        B *= self.expV
        return sfft.irfft(B, n=self.n_p, axis=0, workers=WORKERS)

    def run(self, W, time_steps):
        for _ in range(time_steps):
            W = self.step(W)
        return W
