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

``BlochOracle`` restates the imaginary-time class ``GPU_Wigner2D_GPitaevskii_Bloch``.

``run`` performs ``n`` steps from the normalised initial state and returns the
observables of the state after each step (rows 0 .. n-1) -- the arrays
``Run()`` leaves for ``timeSteps + 1 = n`` steps -- plus the per-step
``ProbabilitySquare_average``.
"""
import dataclasses

import numpy as np

from .common import cuda_f, eval_expr_like, fft, ifft_unnormalised, kernel_coord
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


class BlochOracle(GPitaevskiiOracle):
    """``GPU_Wigner2D_GPitaevskii_Bloch`` (``GPU_Wigner2D_GPitaevskii.py:2064-2545``):
    imaginary-time Strang steps with real exponentials (``Kernel_Bloch`` of
    ``expPotential_source`` :90-114, ``expPLambdaKinetic_source`` :155-178 and
    ``expPotential_GrossPitaevskii_source`` :497-517), normalisation every step,
    and ``Run``'s accept / reject rule: a step counts only if the total energy
    (Hamiltonian K(P) + V(0, X) plus the mean-field energy) falls and
    |purity| < 1, otherwise dt is halved and the previous state restored."""

    def __init__(self, prm: WignerParams, gp_coefficient=0.0):
        super().__init__(prm, gp_coefficient)
        tab, k = self.tab, self.kc
        P = tab.P + 0. * tab.X
        Kp = eval_expr_like(prm.kinetic, P.shape, p=P, cf=prm.cvec())
        V0 = eval_expr_like(prm.potential, tab.X.shape, t=0., x=tab.X, cf=prm.cvec())
        self.H = Kp + V0 + 0. * P
        hb = k['hBar']
        lam = kernel_coord(k['dlambda'], prm.n_x)[np.newaxis, :]
        p = kernel_coord(k['dp'], prm.n_p)[:, np.newaxis]
        self.kin_sum = (eval_expr_like(prm.kinetic, (prm.n_p, prm.n_x), p=p + hb * lam / 2., **k) +
                        eval_expr_like(prm.kinetic, (prm.n_p, prm.n_x), p=p - hb * lam / 2., **k))

    def bloch_half(self, W, t, dtb, gexp):
        k, prm = self.kc, self.prm
        hb = k['hBar']
        shape = (prm.n_p, prm.n_x)
        Vm = eval_expr_like(prm.potential, shape, t=t, x=self.xk - hb * self.thk / 2., **k)
        Vp = eval_expr_like(prm.potential, shape, t=t, x=self.xk + hb * self.thk / 2., **k)
        B = fft(W, 0) * np.exp(-0.25 * dtb * (Vm + Vp))
        if gexp is not None:
            B = B * gexp
        return ifft_unnormalised(B, 0) * (1. / float(prm.n_p))

    def gp_bloch(self, Px, dtb):
        Ph = fft(Px.astype(np.complex128), 0)[np.newaxis, :]
        Bm = ifft_unnormalised(Ph / self.shift, 1) * (1. / float(self.prm.n_x))
        Bp = ifft_unnormalised(Ph * self.shift, 1) * (1. / float(self.prm.n_x))
        return np.exp(-0.25 * dtb * self.a_gp_k * (Bm + Bp))

    def step_bloch(self, W, t, dtb, W0=None):
        prm = self.prm
        ge = self.gp_bloch(self.marginal_x(W), dtb) if self.a_gp != 0. else None
        W = self.bloch_half(W, t, dtb, ge)
        B = fft(W, 1) * np.exp(-0.5 * dtb * self.kin_sum)
        W = ifft_unnormalised(B, 1) * (1. / float(prm.n_x))
        ge = self.gp_bloch(self.marginal_x(W), dtb) if self.a_gp != 0. else None
        W = self.bloch_half(W, t, dtb, ge)
        if W0 is not None:
            c = 2 * np.pi * prm.hbar * prm.dX * prm.dP * np.sum(W * W0)
            W = W - c * W0
        norm = W.sum() * (prm.dX * prm.dP)
        return W / norm

    def stats(self, W):
        prm, tab = self.prm, self.tab
        dXdP = prm.dX * prm.dP
        X, P = tab.X + 0. * tab.P, tab.P + 0. * tab.X
        out = [dXdP * np.sum(W * X), dXdP * np.sum(W * X ** 2), dXdP * np.sum(W * P),
               dXdP * np.sum(W * P ** 2), dXdP * np.sum(W * self.H)]
        purity = 2 * np.pi * prm.hbar * np.sum(W ** 2) * dXdP
        Px = self.marginal_x(W)
        nle = prm.dX * 0.5 * self.a_gp * np.sum(Px ** 2) if self.a_gp != 0. else 0.
        return out, purity, nle

    def run_bloch(self, W_init, time_steps, W0=None):
        """``Run`` (:2105-2342), or with the ground state ``W0`` given
        ``Run_ExitedState1`` (:2343-2545): returns the per-step averages, the
        accepted energies / mean-field energies / purities and the final state.
        The excited-state acceptance also needs a p-marginal dX Re sum_x W with
        no negative value; the reference's ``ProbabilityP`` (:428-441) is meant
        to compute it but strides rows by the row length, so this check is the
        intended one, not the reference's."""
        prm = self.prm
        W = self.initial_normalise(W_init)
        W_step = np.ascontiguousarray(W_init, dtype=np.complex128)
        o, _, nle = self.stats(W)
        energy = o[4] + nle
        dtb = prm.dt
        avg, hist_e, hist_nle, hist_pur = [], [], [], []
        for t_index in range(time_steps + 1):
            W = self.step_bloch(W, t_index * prm.dt, dtb, W0)
            o, purity, nle = self.stats(W)
            avg.append([v.real for v in o])
            e_step = o[4] + nle
            neg_p = W0 is not None and bool(np.any(W.sum(axis=1).real * prm.dX < 0.))
            if t_index > 0:
                if e_step.real < energy.real and abs(purity) < 1. and not neg_p:
                    W_step = W.copy()
                    hist_pur.append(purity.real)
                    hist_e.append(e_step.real)
                    energy = e_step
                    hist_nle.append(np.real(nle))
                else:
                    dtb = dtb / 2.
                    W = W_step.copy()
        return dict(avg=np.array(avg), energy=np.array(hist_e), nle=np.array(hist_nle),
                    purity=np.array(hist_pur), W=W, dt_final=dtb)

