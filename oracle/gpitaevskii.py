"""CPU oracle: restatement of ``GPU_Wigner2D_GPitaevskii.Run`` (TEST INFRASTRUCTURE).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may use
this module.  It restates in numpy (complex128) the Strang-split Wigner step
of ``GPU_Wigner2D_GPitaevskii.py`` with its Gross-Pitaevskii term:

* half potential step ``expPotential_source`` Kernel -- phase
  0.5 dt [V(x - hbar theta/2) - V(x + hbar theta/2)]/hbar, diffusion
  exp(-0.5 D_Theta theta^2 dt), the two absorbing masks
  (``GPU_Wigner2D_GPitaevskii.py:27-88``);
* kinetic step from the kinetic string ``expPLambdaKinetic_source`` Kernel
  (``:117-152``);
* Gross-Pitaevskii factor ``expPotential_GrossPitaevskii_source`` Kernel
  (``:466-495``): with P(x) = dP Re sum_p W (``ProbabilityX`` :1743-1748) and
  B_-+(theta, x) = P(x -+ theta/2) built by ``MakeGrossPitaevskiiTerms``
  (:1717-1736, ``roll_FirstRowCopy_source`` :444-464, the shift phase
  exp(i lambda theta / 2) of ``SetPhaseSpaceGrid2D`` :595-596), the theta-space
  factor exp(i phase), phase = -0.5 dt a_GP Re(B_- - B_+)/hbar;
* the loop (:1897-1990): [GP terms, half potential] -> kinetic -> [GP terms,
  half potential] -> damping (Caldeira-Leggett order 3 or ODM order 1) and, if
  damped, normalisation; observables and sum_x P(x)^2 dx after every step.

``run`` performs ``n`` steps from the normalised initial state and returns the
observables of the state after each step (rows 0 .. n-1) -- the arrays
``Run()`` leaves for ``timeSteps + 1 = n`` steps -- plus the per-step
``ProbabilitySquare_average``.
"""
import dataclasses

import numpy as np

from .common import cuda_f, eval_expr_like, fft, ifft_unnormalised
from .wigner2d import OBS_NAMES, WignerOracle, WignerParams


class GPitaevskiiOracle(WignerOracle):
    def __init__(self, prm: WignerParams, gp_coefficient=0.0):
        # the kinetic factor comes from the kinetic string (expPLambdaKinetic_source), the
        # form WignerOracle builds for GPU_Wigner2D_ODM2; ODM damping is one term, weight 1
        super().__init__(dataclasses.replace(prm, odm2=True, weight1=1., weight2=0.))
        k = self.kc
        self.a_gp = float(gp_coefficient)
        self.a_gp_k = cuda_f(self.a_gp) if prm.constants == 'cuda_%f' else self.a_gp
        self.r_half = np.exp(-0.5 * k['D_Theta'] * self.thk * self.thk * k['dt'])
        # exp(0.5 i Lambda Theta) on the exact host grids (SetPhaseSpaceGrid2D :595-596)
        self.shift = np.exp(0.5j * self.tab.Lambda * self.tab.Theta)

    def half_potential_factor(self, t):
        k, prm = self.kc, self.prm
        hb = k['hBar']
        shape = (prm.n_p, prm.n_x)
        Vm = eval_expr_like(prm.potential, shape, t=t, x=self.xk - hb * self.thk / 2., **k)
        Vp = eval_expr_like(prm.potential, shape, t=t, x=self.xk + hb * self.thk / 2., **k)
        phase = 0.5 * k['dt'] * ((Vm - Vp) / hb)
        r = self.r_half
        return ((r * np.cos(phase)) + 1j * (-r * np.sin(phase))) * self.mask1 * self.mask2

    def marginal_x(self, W):
        """``ProbabilityX``: dP Re sum_p W, per column."""
        return W.sum(axis=0).real * self.prm.dP

    def gp_factor(self, Px):
        """theta-space factor of ``expPotential_GrossPitaevskii_source`` Kernel."""
        k = self.kc
        Ph = fft(Px.astype(np.complex128), 0)[np.newaxis, :]
        Bm = ifft_unnormalised(Ph / self.shift, 1) * (1. / float(self.prm.n_x))
        Bp = ifft_unnormalised(Ph * self.shift, 1) * (1. / float(self.prm.n_x))
        phase = -0.5 * k['dt'] * self.a_gp_k * (Bm - Bp).real / k['hBar']
        return np.cos(phase) + 1j * np.sin(phase)

    def half_step(self, W, t, gp):
        B = fft(W, 0) * self.half_potential_factor(t)
        if gp is not None:
            B = B * gp
        return ifft_unnormalised(B, 0) * (1. / float(self.prm.n_p))

    def step_gp(self, W, t):
        """One iteration of the ``GPU_Wigner2D_GPitaevskii.Run`` loop; returns
        (W, sum_x P(x)^2 dx of the post-kinetic state, or nan without GP)."""
        prm = self.prm
        gp = self.gp_factor(self.marginal_x(W)) if self.a_gp != 0. else None
        W = self.half_step(W, t, gp)
        B = fft(W, 1) * self.kin
        W = ifft_unnormalised(B, 1) * (1. / float(prm.n_x))
        psq = np.nan
        if self.a_gp != 0.:
            Px = self.marginal_x(W)
            psq = float(np.sum(Px ** 2) * prm.dX)
            gp = self.gp_factor(Px)
        W = self.half_step(W, t, gp)
        if prm.gamma != 0.:
            if prm.damping == 'CaldeiraLeggett':
                W = self.caldeira_order3(W)
            if prm.damping == 'ODM':
                W = W + self.lindblad_odm(W, 1., 1.)
            norm = W.sum() * (prm.dX * prm.dP)
            W = W * (1 / norm)
        return W, psq

    def run(self, W_init, n_steps, t_index0=0, normalise_first=True):
        W = self.initial_normalise(W_init) if normalise_first else \
            np.ascontiguousarray(W_init, dtype=np.complex128)
        obs = np.empty((n_steps, len(OBS_NAMES)))
        psq = np.empty(n_steps)
        for n in range(n_steps):
            W, psq[n] = self.step_gp(W, (t_index0 + n) * self.prm.dt)
            obs[n] = self.observables(W)
        return obs, W, psq
