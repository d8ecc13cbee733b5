"""CPU oracle: restatement of ``GPU_Dirac2D.Run`` (TEST INFRASTRUCTURE).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may use
this module.  numpy + ``scipy.fft``, complex128 throughout:

* grids, ``%f`` constants -- ``GPU_Dirac2D.py:306-367``;
* kinetic 4x4 mix ``BaseCUDAsource_K`` -- ``GPU_Dirac2D.py:74-117``;
* mass / 4-potential mix ``DiracPropagatorA_source`` -- ``:123-222``;
* absorbing boundary ``BaseCUDAsource_AbsorbBoundary_xy`` -- ``:225-283``;
* ``Potential_0_Average_source`` -- ``:27-68``;
* observables and normalisations -- ``:776-969``;
* the loop -- ``:973-1133`` (``timeSteps`` propagations at t = dt*t_index,
  t_index = 1..timeSteps, samples taken before each propagation).

Observable columns (``DIRAC_OBS_NAMES``): <x>, <y>, <alpha1>, <alpha2>, <beta>,
<K>, <A0> as the reference's ``Run`` records them; then two columns with no
reference counterpart: <px>, <py> taken in momentum space after
``Normalize_P`` (the reference's ``Average_Px`` weights the x-space density by
the p grid and is never called), and ``norm_kept`` = sum |psi|^2 after / before
the absorbing boundary of the propagation that precedes the sample (1 for the
first sample): the fraction of probability the boundary kept in that step,
which ``Normalize_X`` then restores to 1.
"""
from dataclasses import dataclass, field

import numpy as np

from .common import (cuda_f, shifted_range, kernel_coord_int, eval_expr_like,
                     fft2, ifft2_unnormalised)

DIRAC_OBS_NAMES = ('x', 'y', 'alpha1', 'alpha2', 'beta', 'K', 'A0', 'px', 'py',
                   'norm_kept')


@dataclass
class DiracParams:
    """``GPU_Dirac2D(gridDIM, amplitude, dt, timeSteps, ...)`` plus the attributes
    an instance sets before ``__init__`` (``GPU_Dirac2D.py:306,356-380``)."""
    n_x: int
    n_y: int
    x_amplitude: float
    y_amplitude: float
    dt: float
    mass: float = 1.0
    c: float = 137.036
    hbar: float = 1.0
    A0: str = '0.'
    A1: str = '0.'
    A2: str = '0.'
    A3: str = '0.'
    constants: str = 'cuda_%f'
    coef: tuple = ()       # values of cf[0..7] in the expression strings

    dX: float = field(init=False)
    dY: float = field(init=False)
    dPx: float = field(init=False)
    dPy: float = field(init=False)

    def __post_init__(self):
        # GPU_Dirac2D.py:312-346
        self.dX = 2. * self.x_amplitude / float(self.n_x)
        self.dY = 2. * self.y_amplitude / float(self.n_y)
        self.Px_amplitude = np.pi / self.dX
        self.dPx = 2 * self.Px_amplitude / self.n_x
        self.Py_amplitude = np.pi / self.dY
        self.dPy = 2 * self.Py_amplitude / self.n_y

    def kconst(self):
        c = cuda_f if self.constants == 'cuda_%f' else float
        cv = np.zeros(8)
        cv[:len(self.coef)] = self.coef
        return dict(mass=c(self.mass), c=c(self.c), dt=c(self.dt), dX=c(self.dX),
                    dY=c(self.dY), dPx=c(self.dPx), dPy=c(self.dPy), cf=cv)


class DiracOracle:
    def __init__(self, prm: DiracParams):
        self.prm = prm
        k = self.kc = prm.kconst()
        nx, ny = prm.n_x, prm.n_y
        self.X = shifted_range(prm.x_amplitude, nx)[np.newaxis, :]
        self.Y = shifted_range(prm.y_amplitude, ny)[:, np.newaxis]
        self.Px = np.fft.fftshift(np.linspace(-prm.Px_amplitude, prm.Px_amplitude - prm.dPx,
                                              nx))[np.newaxis, :]
        self.Py = np.fft.fftshift(np.linspace(-prm.Py_amplitude, prm.Py_amplitude - prm.dPy,
                                              ny))[:, np.newaxis]
        # ---- K kernel (GPU_Dirac2D.py:74-117)
        px = kernel_coord_int(k['dPx'], nx)[np.newaxis, :]
        py = kernel_coord_int(k['dPy'], ny)[:, np.newaxis]
        pp = np.sqrt(px * px + py * py + np.power(10., -12))
        cdt = k['c'] * k['dt']
        self.k_sdt = np.sin(cdt * pp) / pp
        self.k_cos = np.cos(cdt * pp) + 0. * px
        self.k_pplus = py + 1j * px
        self.k_pminus = py + 1j * (-px)
        # ---- A kernel geometry (:155-160)
        self.xk = kernel_coord_int(k['dX'], nx)[np.newaxis, :]
        self.yk = kernel_coord_int(k['dY'], ny)[:, np.newaxis]
        self._A_cache = None
        # ---- absorbing boundary (:225-283): j, i are the unshifted indices
        j = ((np.arange(nx) + nx // 2) % nx).astype(np.float64)[np.newaxis, :]
        i = ((np.arange(ny) + ny // 2) % ny).astype(np.float64)[:, np.newaxis]
        wx = np.power(3. * float(nx) / 100., 2)
        wy = np.power(3. * float(ny) / 100., 2)
        self.b1 = 1. - np.exp(-(j * j) / wx)
        self.b2 = 1. - np.exp(-(j - nx + 1.) * (j - nx + 1.) / wx)
        self.b3 = 1. - np.exp(-(i * i) / wy)
        self.b4 = 1. - np.exp(-((i - ny + 1) * (i - ny + 1)) / wy)

    # ------------------------------------------------------------ kernels
    def _A_fields(self, t):
        prm, k = self.prm, self.kc
        shape = (prm.n_y, prm.n_x)
        env = dict(t=t, x=self.xk, y=self.yk, **k)
        return [eval_expr_like(s, shape, **env) for s in (prm.A0, prm.A1, prm.A2, prm.A3)]

    def apply_K(self, P):
        s, cs, pp_, pm_ = self.k_sdt, self.k_cos, self.k_pplus, self.k_pminus
        p1, p2, p3, p4 = P
        return np.array([cs * p1 - (pp_ * s) * p4,
                         cs * p2 + (pm_ * s) * p3,
                         ((-pp_) * s) * p2 + cs * p3,
                         (pm_ * s) * p1 + cs * p4])

    def apply_A(self, P, t):
        k = self.kc
        A0, A1, A2, A3 = self._A_fields(t)
        mass, c, dt = k['mass'], k['c'], k['dt']
        F = np.sqrt(np.power(mass * c * c, 2.) + c * (np.power(A1, 2.) + np.power(A2, 2.)
                                                      + np.power(A3, 2.)))
        expV0 = np.exp((-1j * dt) * A0)
        sn = np.sin(dt * F)
        cs = np.cos(dt * F)
        U11 = cs + 1j * ((-mass) * c * c * sn / F)
        U33 = cs + 1j * (mass * c * c * sn / F)
        U31 = 0. + 1j * (A3 * sn / F)
        U41 = (-A2 * sn / F) + 1j * (A1 * sn / F)
        U32 = (A2 * sn / F) + 1j * (A1 * sn / F)
        U42 = 0. + 1j * (-A3 * sn / F)
        U13, U14, U23, U24, U22, U44 = U31, U32, U41, U42, U11, U33
        p1, p2, p3, p4 = P
        return np.array([expV0 * (U11 * p1 + U13 * p3 + U14 * p4),
                         expV0 * (U22 * p2 + U23 * p3 + U24 * p4),
                         expV0 * (U31 * p1 + U32 * p2 + U33 * p3),
                         expV0 * (U41 * p1 + U42 * p2 + U44 * p4)])

    def apply_boundary(self, P):
        for b in (self.b1, self.b2, self.b3, self.b4):
            P = P * b
        return P

    # ------------------------------------------------------------ observables
    def x_observables(self, P, t):
        prm, k = self.prm, self.kc
        dXdY = prm.dX * prm.dY
        rho = [np.abs(p) ** 2 for p in P]
        x = sum(np.sum(r * self.X) for r in rho) * dXdY
        y = sum(np.sum(r * self.Y) for r in rho) * dXdY
        p1, p2, p3, p4 = P
        a1 = (np.sum(p2 * np.conj(p3)).real + np.sum(p1 * np.conj(p4)).real) * (2. * prm.dX * prm.dY)
        a2 = (-np.sum(p4 * np.conj(p1)) + np.sum(p3 * np.conj(p2)) - np.sum(p2 * np.conj(p3))
              + np.sum(p1 * np.conj(p4))) * (1j * prm.dX * prm.dY)
        beta = (np.sum(p1 * np.conj(p1)) + np.sum(p2 * np.conj(p2)) - np.sum(p3 * np.conj(p3))
                - np.sum(p4 * np.conj(p4))) * dXdY
        A0 = eval_expr_like(prm.A0, (prm.n_y, prm.n_x), t=t, x=self.xk, y=self.yk, **k)
        a0 = prm.dX * prm.dY * np.sum(A0 * rho[0] + A0 * rho[1] + A0 * rho[2] + A0 * rho[3])
        return [x.real, y.real, a1, a2.real, beta.real, a0.real]

    def p_observables(self, Q):
        prm = self.prm
        q1, q2, q3, q4 = Q
        dd = prm.dPx * prm.dPy
        e = (np.sum(q1 * np.conj(q1)) + np.sum(q2 * np.conj(q2)) - np.sum(q3 * np.conj(q3))
             - np.sum(q4 * np.conj(q4)))
        e = e * (prm.mass * prm.c * prm.c * prm.dPx * prm.dPy)
        t1 = (q4 * np.conj(q1) + q1 * np.conj(q4) + q3 * np.conj(q2) + q2 * np.conj(q3)) * self.Px
        e = e + np.sum(t1) * prm.dPx * prm.dPy * prm.c
        t2 = (q4 * np.conj(q1) - q1 * np.conj(q4) - q3 * np.conj(q2) + q2 * np.conj(q3)) * self.Py
        e = e + np.sum(t2) * prm.dPx * prm.dPy * prm.c * (-1j)
        rho = sum(np.abs(q) ** 2 for q in Q)
        px = np.sum(rho * self.Px) * dd
        py = np.sum(rho * self.Py) * dd
        return e.real, px.real, py.real

    def norm_x(self, P):
        s = sum(np.sum(np.abs(p) ** 2) for p in P)
        return np.sqrt(s * self.prm.dX * self.prm.dY), s * self.prm.dX * self.prm.dY

    def norm_p(self, Q):
        s = sum(np.sum(np.abs(q) ** 2) for q in Q)
        return np.sqrt(s * self.prm.dPx * self.prm.dPy)

    # ------------------------------------------------------------ loop
    def run(self, psi_init, n_steps, record_final=False):
        """``GPU_Dirac2D.Run`` with ``timeSteps = n_steps``.  Returns
        (obs[n_steps (+1 if record_final), 10], psi_end[4, ny, nx])."""
        prm = self.prm
        P = np.ascontiguousarray(psi_init, dtype=np.complex128).copy()
        nrm, _ = self.norm_x(P)
        P = P * (1 / nrm)
        kept = 1.0
        n_rec = n_steps + (1 if record_final else 0)
        obs = np.zeros((n_rec, len(DIRAC_OBS_NAMES)))
        inv = 1. / float(prm.n_x * prm.n_y)
        for t_index in range(1, n_steps + 1):
            t = np.float64(prm.dt * t_index)
            xo = self.x_observables(P, t)
            Q = fft2(P)
            Q = Q * (1 / self.norm_p(Q))
            K, px, py = self.p_observables(Q)
            obs[t_index - 1] = xo[:5] + [K, xo[5], px, py, kept]
            Q = self.apply_K(Q)
            P = ifft2_unnormalised(Q) * inv
            P = self.apply_A(P, t)
            _, before = self.norm_x(P)
            P = self.apply_boundary(P)
            nrm, after = self.norm_x(P)
            kept = after / before
            P = P * (1 / nrm)
        if record_final:
            t = np.float64(prm.dt * (n_steps + 1))
            xo = self.x_observables(P, t)
            Q = fft2(P)
            Q = Q * (1 / self.norm_p(Q))
            K, px, py = self.p_observables(Q)
            obs[n_steps] = xo[:5] + [K, xo[5], px, py, kept]
        return obs, P


def spinor_particle_spin_up(prm: DiracParams, p_init, modulation):
    """``Spinor_Particle_SpinUp`` (``GPU_Dirac2D.py:419-434``), shifted layout."""
    X = shifted_range(prm.x_amplitude, prm.n_x)[np.newaxis, :]
    Y = shifted_range(prm.y_amplitude, prm.n_y)[:, np.newaxis]
    px, py = p_init
    rho = np.exp(1j * X * px + 1j * Y * py) * modulation(X, Y)
    p0 = np.sqrt(px * px + py * py + (prm.mass * prm.c) ** 2)
    return np.array([rho * (p0 + prm.mass * prm.c), rho * 0., rho * 0., rho * (px + 1j * py)])
