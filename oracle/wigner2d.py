"""CPU oracle: restatement of ``GPU_Wigner2D_FFT.Run`` (TEST INFRASTRUCTURE).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may use
this module.  It restates, in numpy + ``scipy.fft`` (complex128 throughout),
the reference's Wigner2D split-operator loop:

* grids and shifted tables -- ``GPU_Wigner2D_FFT.py:549-595``;
* ``%f`` kernel constants -- ``GPU_Wigner2D_FFT.py:833-842``;
* kinetic phase ``expPLambda_source`` -- ``GPU_Wigner2D_FFT.py:131-158``,
  or ``expPLambdaKinetic_source`` -- ``:162-200`` (used by ``GPU_Wigner2D_ODM2``);
* Moyal potential phase + absorbing mask ``expPotential_source`` -- ``:80-126``;
* Caldeira-Leggett ``theta_fp_source`` / ``Theta_fp_Damping`` /
  ``CaldeiraDissipatorOrder3`` -- ``:399-431,1135-1157``;
* ODM Lindblad ``g_ODM`` / ``SetA_ODM`` / ``_Lindbladian_ODM`` /
  ``Lindbladian_ODM_Order1`` -- ``:1196-1244,1516-1643``;
* the loop, observables and normalisation -- ``:1754-1934`` (and the ODM2
  variant ``:2060-2176``).

Loop convention: :func:`run` performs ``n_prop`` propagations and returns
``n_prop + 1`` observable samples (sample k is taken before propagation k; the
last one after the final propagation).  The reference's ``Run()`` performs
``timeSteps + 1`` propagations and keeps the first ``timeSteps + 1`` samples
(``GPU_Wigner2D_FFT.py:1776,1843``).

Observable columns (``OBS_NAMES``): norm, <x>, <x^2>, <p>, <p^2>, <xp>, <V'>,
<pV'>, <xV'>, <H>, negative area.  The reference records all but ``norm``
(``GPU_Wigner2D_FFT.py:1857-1878``); ``norm`` = dX dP Re(sum W) of the sampled W.
"""
import re
from dataclasses import dataclass, field

import numpy as np

from .common import (cuda_f, shifted_range, kernel_coord, eval_expr_like,
                     fft, ifft_unnormalised)

OBS_NAMES = ('norm', 'x', 'x2', 'p', 'p2', 'xp', 'dV', 'pdV', 'xdV', 'H',
             'negative_area')


@dataclass
class WignerParams:
    """Constructor arguments of ``GPU_Wigner2D_FFT`` (``GPU_Wigner2D_FFT.py:1718``)
    plus the attributes instances set before ``__init__`` (``SetTimeTrack``,
    ``dampingFunction``, ``fp_Damping_String``, ``epsilon``, ``L_material``)."""
    n_x: int
    n_p: int
    x_amplitude: float
    p_amplitude: float
    dt: float
    hbar: float = 1.0
    mass: float = 1.0
    d_theta: float = 0.0
    d_lambda: float = 0.0
    gamma: float = 0.0
    potential: str = '0.5*pow(x,2)'
    dpotential: str = 'x'
    kinetic: str = '0.5*p*p'
    damping: str = 'CaldeiraLeggett'       # 'CaldeiraLeggett' | 'ODM' | other
    fp_damping: str = 'fabs(p)'
    epsilon: float = 0.5
    L_material: float = 1.0
    # GPU_Wigner2D_ODM2: kinetic from the kinetic string, two Lindblad terms
    odm2: bool = False
    weight1: float = 1.0
    weight2: float = 0.0
    constants: str = 'cuda_%f'             # 'cuda_%f' | 'exact'
    coef: tuple = ()                       # values of cf[0..7] in the expression strings
    # GPU_FokkerPlank2D_FFT (GPU_Wigner2D_FFT.py:2242-2459): the classical (KvN /
    # Liouville) potential factor exp(+i dt V'(t, x) theta) instead of the Moyal one
    # (exp_PotentialKvN_source :27-75), and its `normalization` argument: damped
    # steps renormalise only when it is 'Wigner' (:2404-2406)
    kvn: bool = False
    normalization: str = 'Wigner'

    # derived (filled by __post_init__)
    dX: float = field(init=False)
    dP: float = field(init=False)
    dTheta: float = field(init=False)
    dLambda: float = field(init=False)

    def __post_init__(self):
        # GPU_Wigner2D_FFT.py:549-563
        self.dX = 2. * self.x_amplitude / float(self.n_x)
        self.dP = 2. * self.p_amplitude / float(self.n_p)
        self.dTheta = 2. * np.pi / (2. * self.p_amplitude)
        self.dLambda = 2. * np.pi / (2. * self.x_amplitude)

    # ---- constants as the kernels see them (GPU_Wigner2D_FFT.py:833-842)
    def kconst(self):
        c = cuda_f if self.constants == 'cuda_%f' else float
        return dict(dt=c(self.dt), dx=c(self.dX), dp=c(self.dP),
                    dtheta=c(self.dTheta), dlambda=c(self.dLambda),
                    mass=c(self.mass), hBar=c(self.hbar),
                    D_Theta=c(self.d_theta), D_Lambda=c(self.d_lambda), cf=self.cvec())

    def cvec(self):
        v = np.zeros(8)
        v[:len(self.coef)] = self.coef
        return v


class Tables:
    """Host tables of ``SetPhaseSpaceGrid2D`` and ``Run`` (exact doubles)."""

    def __init__(self, prm: WignerParams):
        self.prm = prm
        nx, npp = prm.n_x, prm.n_p
        Theta_amplitude = prm.dTheta * npp / 2.
        Lambda_amplitude = prm.dLambda * nx / 2.
        # GPU_Wigner2D_FFT.py:568-581
        self.X = shifted_range(prm.x_amplitude, nx)[np.newaxis, :]
        self.P = shifted_range(prm.p_amplitude, npp)[:, np.newaxis]
        self.Theta = np.fft.fftshift(np.linspace(-Theta_amplitude, Theta_amplitude - prm.dTheta,
                                                 npp))[:, np.newaxis]
        self.Lambda = np.fft.fftshift(np.linspace(-Lambda_amplitude, Lambda_amplitude - prm.dLambda,
                                                  nx))[np.newaxis, :]
        shape = (npp, nx)
        # observable tables, GPU_Wigner2D_FFT.py:583-591,1747,1785-1792
        dV = eval_expr_like(prm.dpotential, self.X.shape, t=0., x=self.X, cf=prm.cvec())
        V0 = eval_expr_like(prm.potential, self.X.shape, t=0., x=self.X, cf=prm.cvec())
        self.dV_x = dV[0].copy()
        self.V0_x = V0[0].copy()
        self.obs_tables = [
            self.X + 0. * self.P,
            self.X ** 2 + 0. * self.P,
            self.P + 0. * self.X,
            self.P ** 2 + 0. * self.X,
            self.P * self.X,
            dV + 0. * self.P,
            self.P * dV,
            dV * self.X + 0. * self.P,
            self.P ** 2 / (2. * prm.mass) + V0,
        ]
        for t in self.obs_tables:
            assert t.shape == shape


def _has_t(expr):
    return re.search(r'(?<![A-Za-z_0-9])t(?![A-Za-z_0-9])', expr) is not None


class WignerOracle:
    """Stateful restatement of one ``GPU_Wigner2D_FFT`` instance."""

    def __init__(self, prm: WignerParams):
        self.prm = prm
        self.tab = Tables(prm)
        k = self.kc = prm.kconst()
        nx, npp = prm.n_x, prm.n_p
        # ---- kinetic factor (expPLambda_source :131-158 / expPLambdaKinetic :162-200)
        lam = kernel_coord(k['dlambda'], nx)[np.newaxis, :]
        p = kernel_coord(k['dp'], npp)[:, np.newaxis]
        if prm.odm2:
            hb = k['hBar']
            Kp = eval_expr_like(prm.kinetic, (npp, nx), p=p + hb * lam / 2., **k)
            Km = eval_expr_like(prm.kinetic, (npp, nx), p=p - hb * lam / 2., **k)
            phase = k['dt'] * ((Kp - Km) / hb)
        else:
            phase = k['dt'] * lam * p / k['mass']
        r = np.exp(-k['D_Lambda'] * lam * lam)
        self.kin = (r * np.cos(phase)) + 1j * (-r * np.sin(phase))
        # ---- potential factor pieces (expPotential_source :80-126)
        self.xk = kernel_coord(k['dx'], nx)[np.newaxis, :]
        self.thk = kernel_coord(k['dtheta'], npp)[:, np.newaxis]
        self.r_theta = np.exp(-k['D_Theta'] * self.thk * self.thk * k['dt'])
        x_max = k['dx'] * (nx - 1.) / 2.
        self.mask1 = 1. - np.exp(-np.power(self.xk - x_max, 2) / np.power(10. * k['dx'], 2))
        self.mask2 = 1. - np.exp(-np.power(self.xk + x_max, 2) / np.power(10. * k['dx'], 2))
        self._pot_cache = None
        self._pot_time_dependent = _has_t(prm.dpotential if prm.kvn else prm.potential)
        # ---- Caldeira-Leggett sign(p) f(p) (theta_fp_source :399-431)
        fp = eval_expr_like(prm.fp_damping, p.shape, p=p, **k)
        self.sfp = np.where(p >= 0., fp, -fp)
        # ---- ODM tables (SetA_ODM :1206-1244)
        if prm.damping == 'ODM':
            self._set_odm()

    # ------------------------------------------------------------ pieces
    def potential_factor(self, t):
        if self._pot_cache is not None and not self._pot_time_dependent:
            return self._pot_cache
        k, prm = self.kc, self.prm
        hb = k['hBar']
        shape = (prm.n_p, prm.n_x)
        if prm.kvn:
            # Potential_XTheta = -dPotential(t, x) theta; phase = dt Potential_XTheta (:41-63)
            dV = eval_expr_like(prm.dpotential, shape, t=t, x=self.xk + 0. * self.thk, **k)
            phase = k['dt'] * (-dV * self.thk)
        else:
            Vm = eval_expr_like(prm.potential, shape, t=t, x=self.xk - hb * self.thk / 2., **k)
            Vp = eval_expr_like(prm.potential, shape, t=t, x=self.xk + hb * self.thk / 2., **k)
            phase = k['dt'] * ((Vm - Vp) / hb)
        r = self.r_theta
        f = (r * np.cos(phase)) + 1j * (-r * np.sin(phase))
        self._pot_cache = f
        return f

    def theta_fp_damping(self, W):
        """``Theta_fp_Damping`` (:1135-1143): IFFT_p[Theta * FFT_p(sign(p) f(p) W)]/N_p."""
        L = W * self.sfp
        L = fft(L, 0)
        L = L * (self.tab.Theta + 0. * self.tab.X)
        L = ifft_unnormalised(L, 0) * (1. / float(self.prm.n_p))
        return L

    def caldeira_order3(self, W):
        """``CaldeiraDissipatorOrder3`` (:1145-1157): W + a(1+a/2)(1+a/3)W,
        a = 2 i gamma dt D (with D = ``Theta_fp_Damping``)."""
        prm = self.prm
        c1 = 2. / 3. * 1j * prm.dt * prm.gamma
        c2 = 2. / 2. * 1j * prm.dt * prm.gamma
        c3 = 2. * 1j * prm.dt * prm.gamma
        LW = W.copy()
        LW = LW + c1 * self.theta_fp_damping(W)
        LW = LW + c2 * self.theta_fp_damping(LW)
        return W + c3 * self.theta_fp_damping(LW)

    def _set_odm(self):
        prm, tab = self.prm, self.tab
        hb, L = prm.hbar, prm.L_material
        X, Th, P, Lam = tab.X, tab.Theta, tab.P, tab.Lambda

        def g(p):                     # g_ODM :1196-1197
            return np.sqrt(L * eval_expr_like(prm.fp_damping, np.shape(p),
                                              p=np.abs(p) + hb / (2. * L), cf=prm.cvec()))

        def gs(p):                    # g_sign_ODM :1199-1200
            return g(p) * np.sign(p)
        Xp = X + 0.5 * hb * Th
        Xm = X - 0.5 * hb * Th
        X0 = X + 0. * Th
        X2 = X + hb * Th
        self.cos_ = np.cos(X0)
        self.cos_plus2 = np.cos(X2)
        self.cos_plus = np.cos(Xp)
        self.cos_minus = np.cos(Xm)
        self.cos_plus_minus = np.cos(Xp) * np.cos(Xm)
        self.sin_ = np.sin(X0)
        self.sin_plus2 = np.sin(X2)
        self.sin_plus = np.sin(Xp)
        self.sin_minus = np.sin(Xm)
        self.sin_plus_minus = np.sin(Xp) * np.sin(Xm)
        pp = P + 0.5 * hb * Lam
        pm = P - 0.5 * hb * Lam
        self.g_plus = g(pp)
        self.g_minus = g(pm)
        self.gg_plus = -0.5 * self.g_plus ** 2
        self.gg_minus = -0.5 * self.g_minus ** 2
        self.g_sign_plus = gs(pp)
        self.g_sign_minus = gs(pm)

    def lindblad_odm(self, W, weight, sign, n=1.):
        """``_Lindbladian_ODM`` (:1516-1634), first order (``Lindbladian_ODM_Order1``
        :1637-1643 adds the result to W)."""
        nx, npp = self.prm.n_x, self.prm.n_p
        Bx = fft(W, 1)

        def x_leg(*tabs):
            T = Bx
            for tb in tabs:
                T = T * tb
            T = ifft_unnormalised(T, 1) * (1. / float(nx))
            return fft(T, 0)
        LW = x_leg(self.g_plus, self.g_minus) * self.cos_plus_minus
        LW = LW + ((x_leg(self.g_plus, self.g_sign_minus) * self.cos_minus) * self.sin_plus) * (1j * sign)
        LW = LW + ((x_leg(self.g_sign_plus, self.g_minus) * self.sin_minus) * self.cos_plus) * (-1j * sign)
        LW = LW + x_leg(self.g_sign_plus, self.g_sign_minus) * self.sin_plus_minus
        LW = LW + x_leg(self.gg_plus)
        LW = LW + x_leg(self.gg_minus)
        LW = ifft_unnormalised(LW, 0) * (1. / float(npp))
        LW = LW * (self.prm.dt * 2 * self.prm.gamma * weight / n)
        return LW

    # ------------------------------------------------------------ step / obs
    def observables(self, W):
        prm, tab = self.prm, self.tab
        dXdP = prm.dX * prm.dP
        out = np.empty(len(OBS_NAMES))
        out[0] = (dXdP * W.sum()).real
        for i, t in enumerate(tab.obs_tables):
            out[1 + i] = (dXdP * np.sum(W * t)).real
        out[10] = (np.sum(np.where(W.real < 0., W, 0.)) * dXdP).real
        return out

    def step(self, W, t):
        """One propagation of the loop body (``GPU_Wigner2D_FFT.py:1884-1913``)."""
        prm = self.prm
        B = fft(W, 1)
        B = B * self.kin
        W = ifft_unnormalised(B, 1) * (1. / float(prm.n_x))
        B = fft(W, 0)
        B = B * self.potential_factor(t)
        B = B * self.mask1
        B = B * self.mask2
        W = ifft_unnormalised(B, 0) * (1. / float(prm.n_p))
        if prm.gamma != 0.:
            if prm.damping == 'CaldeiraLeggett':
                W = self.caldeira_order3(W)
            if prm.damping == 'ODM':
                if prm.odm2:
                    W = W + self.lindblad_odm(W, prm.weight1, 1.)
                    W = W + self.lindblad_odm(W, prm.weight2, -1.)
                else:
                    W = W + self.lindblad_odm(W, 1., 1.)
            if not prm.kvn or prm.normalization == 'Wigner':
                norm = W.sum() * (prm.dX * prm.dP)
                W = W * (1 / norm)
        return W

    def initial_normalise(self, W_init):
        """``Run`` prologue (:1778-1780): W /= sum(W) dX dP."""
        W = np.ascontiguousarray(W_init, dtype=np.complex128)
        norm = W.sum() * self.prm.dX * self.prm.dP
        return W * (1 / norm)

    def run(self, W_init, n_prop, t_index0=0, normalise_first=True):
        """``n_prop`` propagations; returns (obs[n_prop+1, 11], W)."""
        W = self.initial_normalise(W_init) if normalise_first else \
            np.ascontiguousarray(W_init, dtype=np.complex128)
        obs = np.empty((n_prop + 1, len(OBS_NAMES)))
        for n in range(n_prop):
            obs[n] = self.observables(W)
            W = self.step(W, (t_index0 + n) * self.prm.dt)
        obs[n_prop] = self.observables(W)
        return obs, W


def run_reference_convention(prm, W_init, time_steps):
    """What ``GPU_Wigner2D_FFT.Run`` returns for ``timeSteps=time_steps``:
    ``time_steps + 1`` propagations, ``time_steps + 1`` samples, ``W_end`` real."""
    o = WignerOracle(prm)
    obs, W = o.run(W_init, time_steps + 1)
    return obs[:time_steps + 1], W


# ---------------------------------------------------------------- initial states
def wigner_harmonic_oscillator(prm, n, omega, x, p):
    """``Wigner_HarmonicOscillator`` (:715-728), shifted layout, normalised."""
    from scipy.special import eval_laguerre
    tab = Tables(prm)
    r2 = prm.mass * omega ** 2 * ((tab.X - x)) ** 2 + ((tab.P - p)) ** 2 / prm.mass
    W = (-1) ** n * eval_laguerre(n, 2 * r2) * np.exp(-r2)
    norm = np.sum(W) * prm.dX * prm.dP
    return W / norm


def wigner_cat_state(prm, x0=3.0, sigma=0.7):
    """Cat state psi ~ g(x-x0) + g(x+x0), g = exp(-x^2/(2 sigma^2)), built with the
    reference's discrete Wigner-transform recipe (``Wigner_Half_HarmonicOscillator``
    :743-771): psi(x - hbar theta/2) psi*(x + hbar theta/2), then IFFT over theta."""
    tab = Tables(prm)
    Theta_amplitude = prm.dTheta * prm.n_p / 2.
    X_range = np.linspace(-prm.x_amplitude, prm.x_amplitude - prm.dX, prm.n_x)
    Theta_range = np.linspace(-Theta_amplitude, Theta_amplitude - prm.dTheta, prm.n_p)

    def psi(x):
        return np.exp(-(x - x0) ** 2 / (2 * sigma ** 2)) + np.exp(-(x + x0) ** 2 / (2 * sigma ** 2))
    Xm = X_range[np.newaxis, :] - 0.5 * prm.hbar * Theta_range[:, np.newaxis]
    Xp = X_range[np.newaxis, :] + 0.5 * prm.hbar * Theta_range[:, np.newaxis]
    W = psi(Xm) * np.conj(psi(Xp))
    W = np.fft.ifft(np.fft.fftshift(W), axis=0)
    norm = np.sum(W) * prm.dX * prm.dP
    W = (W / norm).real
    del tab
    return np.ascontiguousarray(W)
