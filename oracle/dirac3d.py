"""CPU oracle: restatement of ``GPU_Dirac3D.Run`` (TEST INFRASTRUCTURE).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may use
this module.  numpy + ``scipy.fft``, complex128, arrays (Z, Y, X) with x
contiguous and every axis FFT-shifted (``GPU_Dirac3D.py:659-661``):

* grids and ``%f`` constants -- ``GPU_Dirac3D.py:634-704``;
* kinetic 4x4 mix ``DiracPropagatorK_source`` -- ``:386-452`` (half the mass:
  ``mass_ = 0.5*mass``, no regularisation of |p|);
* mass / 4-potential mix ``DiracPropagatorA_source`` -- ``:455-559`` (the other
  half of the mass; F = sqrt((mass_ c^2)^2 + A1^2 + A2^2 + A3^2));
* position averages ``Average_X/Y/Z_source`` (``:264-383``), ``Average_Alpha1/2/3``
  (``:1221-1249``), ``Potential_0_Average_source`` (``:92-138``); momentum
  averages ``Average_Px/Py/Pz_source`` (``:142-261``) and ``K_Energy_Average_source``
  (``:27-89``) on the spectrum divided by the momentum-space norm of step 1;
* the loop ``Run`` -- ``:1265-1500``: one ``Normalize_GPU`` before the loop, then
  for t_index = 1..timeSteps (t = dt t_index): position averages, FFT,
  [momentum averages], K, IFFT / N, A(t).  No boundary, no renormalisation.

The reference's 3-D plan is ``cufftPlanMany(3, [X, Y, Z])`` on (Z, Y, X) arrays,
which is the transform of the arrays as laid out only when X == Z; this oracle
transforms the arrays as laid out (equal to the reference on cubic grids).

Observable columns (``DIRAC3D_OBS_NAMES``): <x>, <y>, <z>, <alpha1>, <alpha2>,
<alpha3>, <A0>, <px>, <py>, <pz>, <K> as ``Run`` records them (samples before
each propagation), then ``norm`` = sum |psi|^2 dX dY dZ of the sample (no
reference counterpart).
"""
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft

from .common import WORKERS, cuda_f, eval_expr_like, kernel_coord_int, shifted_range

DIRAC3D_OBS_NAMES = ('x', 'y', 'z', 'alpha1', 'alpha2', 'alpha3', 'A0', 'px', 'py', 'pz', 'K', 'norm')


@dataclass
class Dirac3DParams:
    """``GPU_Dirac3D(gridDIM, amplitude, dt, timeSteps, ...)`` plus the attributes an
    instance sets before ``__init__`` (``mass``, ``c``, ``hBar``,
    ``Potential_{0..3}_String`` as C expressions in (t, x, y, z))."""
    n_x: int
    n_y: int
    n_z: int
    x_amplitude: float
    y_amplitude: float
    z_amplitude: float
    dt: float
    mass: float = 1.0
    c: float = 137.036
    hbar: float = 1.0
    A0: str = '0.'
    A1: str = '0.'
    A2: str = '0.'
    A3: str = '0.'
    constants: str = 'cuda_%f'
    coef: tuple = ()

    dX: float = field(init=False)
    dY: float = field(init=False)
    dZ: float = field(init=False)
    dPx: float = field(init=False)
    dPy: float = field(init=False)
    dPz: float = field(init=False)

    def __post_init__(self):
        # GPU_Dirac3D.py:637-683
        self.dX = 2. * self.x_amplitude / float(self.n_x)
        self.dY = 2. * self.y_amplitude / float(self.n_y)
        self.dZ = 2. * self.z_amplitude / float(self.n_z)
        self.dPx = 2 * (np.pi / self.dX) / self.n_x
        self.dPy = 2 * (np.pi / self.dY) / self.n_y
        self.dPz = 2 * (np.pi / self.dZ) / self.n_z

    def kconst(self):
        c = cuda_f if self.constants == 'cuda_%f' else float
        cv = np.zeros(8)
        cv[:len(self.coef)] = self.coef
        return dict(hBar=c(self.hbar), mass=c(self.mass), c=c(self.c), dt=c(self.dt), dX=c(self.dX),
                    dY=c(self.dY), dZ=c(self.dZ), dPx=c(self.dPx), dPy=c(self.dPy), dPz=c(self.dPz), cf=cv)


def fftn3(a):
    return sfft.fftn(a, axes=(-3, -2, -1), workers=WORKERS)


def ifftn3_unnormalised(a):
    return sfft.ifftn(a, axes=(-3, -2, -1), norm='forward', workers=WORKERS)


class Dirac3DOracle:
    def __init__(self, prm: Dirac3DParams):
        self.prm = prm
        k = self.kc = prm.kconst()
        nx, ny, nz = prm.n_x, prm.n_y, prm.n_z
        self.shape = (nz, ny, nx)
        # kernel coordinates (every kernel: j = (idx + N/2) % N, x = dX (j - N/2))
        self.xk = kernel_coord_int(k['dX'], nx)[np.newaxis, np.newaxis, :]
        self.yk = kernel_coord_int(k['dY'], ny)[np.newaxis, :, np.newaxis]
        self.zk = kernel_coord_int(k['dZ'], nz)[:, np.newaxis, np.newaxis]
        self.px = kernel_coord_int(k['dPx'], nx)[np.newaxis, np.newaxis, :]
        self.py = kernel_coord_int(k['dPy'], ny)[np.newaxis, :, np.newaxis]
        self.pz = kernel_coord_int(k['dPz'], nz)[:, np.newaxis, np.newaxis]
        # ---- K mix (DiracPropagatorK_source :410-446)
        mass_, c, dt, hb = 0.5 * k['mass'], k['c'], k['dt'], k['hBar']
        px, py, pz = self.px, self.py, self.pz
        E = c * np.sqrt(px * px + py * py + pz * pz + np.power(mass_ * c, 2))
        phi = E * dt / hb
        sn, cs = np.sin(phi), np.cos(phi)
        self.U11 = cs + 1j * (-c * c * mass_ * sn / E)
        self.U33 = cs + 1j * (c * c * mass_ * sn / E)
        pplus, pminus = py + 1j * px, py - 1j * px
        self.U13 = 0. + 1j * (-c * pz * sn / E)
        self.U14 = -pplus * c * sn / E
        self.U23 = (c * sn / E) * pminus
        self.U24 = 0. + 1j * (c * pz * sn / E)
        self.U31 = 0. + 1j * (-c * pz * sn / E)
        self.U32 = -(c * sn / E) * pplus
        self.U41 = pminus * (c * sn / E)
        self.U42 = 0. + 1j * (c * pz * sn / E)
        self.s1 = None            # momentum-space norm of step 1 (:1396-1398)

    def _fields(self, t):
        prm, k = self.prm, self.kc
        env = dict(t=t, x=self.xk, y=self.yk, z=self.zk, **k)
        return [eval_expr_like(s, self.shape, **env) for s in (prm.A0, prm.A1, prm.A2, prm.A3)]

    def apply_K(self, Q):
        q1, q2, q3, q4 = Q
        return np.array([self.U11 * q1 + self.U13 * q3 + self.U14 * q4,
                         self.U11 * q2 + self.U23 * q3 + self.U24 * q4,
                         self.U31 * q1 + self.U32 * q2 + self.U33 * q3,
                         self.U41 * q1 + self.U42 * q2 + self.U33 * q4])

    def apply_A(self, P, t):
        k = self.kc
        A0, A1, A2, A3 = self._fields(t)
        mass_, c, dt, hb = 0.5 * k['mass'], k['c'], k['dt'], k['hBar']
        F = np.sqrt(np.power(mass_ * c * c, 2.) + (np.power(A1, 2.) + np.power(A2, 2.) + np.power(A3, 2.)))
        om = F / hb
        sn, cs = np.sin(dt * om), np.cos(dt * om)
        iA_plus, iA_minus = -A2 + 1j * A1, A2 + 1j * A1
        e = np.exp(0. + 1j * (-dt * A0))
        U11 = cs + 1j * (-mass_ * c * c * sn / F)
        U33 = cs + 1j * (mass_ * c * c * sn / F)
        U13 = 0. + 1j * (A3 * sn / F)
        U14 = iA_minus * sn / F
        U23 = iA_plus * sn / F
        U24 = 0. + 1j * (-A3 * sn / F)
        p1, p2, p3, p4 = P
        return np.array([e * (U11 * p1 + U13 * p3 + U14 * p4),
                         e * (U11 * p2 + U23 * p3 + U24 * p4),
                         e * (U13 * p1 + U14 * p2 + U33 * p3),
                         e * (U23 * p1 + U24 * p2 + U33 * p4)])

    # ------------------------------------------------------------ observables
    def x_observables(self, P, t):
        prm, k = self.prm, self.kc
        dV = prm.dX * prm.dY * prm.dZ
        rho = sum(np.abs(p) ** 2 for p in P)
        x = np.sum(rho * self.xk) * prm.dX * prm.dY * prm.dZ
        y = np.sum(rho * self.yk) * prm.dX * prm.dY * prm.dZ
        z = np.sum(rho * self.zk) * prm.dX * prm.dY * prm.dZ
        p1, p2, p3, p4 = P
        dot = lambda a, b: np.sum(a * np.conj(b))
        a1 = (dot(p4, p1) + dot(p3, p2) + dot(p2, p3) + dot(p1, p4)) * dV
        a2 = (-dot(p4, p1) + dot(p3, p2) - dot(p2, p3) + dot(p1, p4)) * (1j * dV)
        a3 = (dot(p3, p1) - dot(p4, p2) + dot(p1, p3) - dot(p2, p4)) * dV
        A0 = eval_expr_like(prm.A0, self.shape, t=t, x=self.xk, y=self.yk, z=self.zk, **k)
        a0 = np.sum(A0 * rho) * prm.dX * prm.dY * prm.dZ
        return [x, y, z, a1.real, a2.real, a3.real, a0, np.sum(rho) * dV]

    def p_observables(self, Q):
        prm, k = self.prm, self.kc
        dP = prm.dPx * prm.dPy * prm.dPz
        S = sum(np.sum(np.abs(q) ** 2) for q in Q)
        if self.s1 is None:
            self.s1 = S
        inv = 1. / (self.s1 * dP)                      # |psi / norm|^2 = |psi|^2 / (S1 dP)
        rho = sum(np.abs(q) ** 2 for q in Q) * inv
        q1, q2, q3, q4 = Q
        re = lambda a, b: (a * np.conj(b)).real
        im = lambda a, b: (a * np.conj(b)).imag
        m, c = k['mass'], k['c']
        w = m * c * c * (np.abs(q1) ** 2 + np.abs(q2) ** 2 - np.abs(q3) ** 2 - np.abs(q4) ** 2)
        w = w + 2 * c * self.px * (re(q4, q1) + re(q3, q2))
        w = w + 2 * c * self.py * (im(q4, q1) + im(q2, q3))
        w = w + 2 * c * self.pz * (re(q3, q1) - re(q4, q2))
        return [np.sum(rho * self.px) * dP, np.sum(rho * self.py) * dP, np.sum(rho * self.pz) * dP,
                np.sum(w * inv) * dP]

    def norm(self, P):
        return np.sqrt(sum(np.sum(np.abs(p) ** 2) for p in P) * self.prm.dX * self.prm.dY * self.prm.dZ)

    # ------------------------------------------------------------ loop
    def run(self, psi_init, n_steps, t_index0=0, normalise=True):
        """``Run`` with ``timeSteps = n_steps`` (``t_index0`` > 0 and
        ``normalise=False`` continue an earlier run, keeping the step-1 norm):
        returns (obs[n_steps, 12], psi_end)."""
        prm = self.prm
        P = np.ascontiguousarray(psi_init, dtype=np.complex128).copy()
        if normalise:
            P = P * (1. / self.norm(P))
        obs = np.zeros((n_steps, len(DIRAC3D_OBS_NAMES)))
        n3 = float(prm.n_x * prm.n_y * prm.n_z)
        for n in range(n_steps):
            t = np.float64(prm.dt * (t_index0 + n + 1))
            xo = self.x_observables(P, t)
            Q = np.array([fftn3(p) for p in P])
            po = self.p_observables(Q)
            obs[n] = xo[:7] + po + [xo[7]]
            Q = self.apply_K(Q)
            P = np.array([ifftn3_unnormalised(q) for q in Q]) * (1. / n3)
            P = self.apply_A(P, t)
        return obs, P


def spinor_grids(prm: Dirac3DParams):
    X = shifted_range(prm.x_amplitude, prm.n_x)[np.newaxis, np.newaxis, :]
    Y = shifted_range(prm.y_amplitude, prm.n_y)[np.newaxis, :, np.newaxis]
    Z = shifted_range(prm.z_amplitude, prm.n_z)[:, np.newaxis, np.newaxis]
    return X, Y, Z


def spinor_particle_spin_up_3d(prm: Dirac3DParams, p_init, modulation):
    """``Spinor_Particle_SpinUp`` (``GPU_Dirac3D.py:787-802``), shifted layout."""
    X, Y, Z = spinor_grids(prm)
    px, py, pz = p_init
    rho = np.exp(1j * px * X + 1j * py * Y + 1j * pz * Z) * modulation(X, Y, Z)
    p0 = np.sqrt(px * px + py * py + pz * pz + (prm.mass * prm.c) ** 2)
    return np.array([rho * (p0 + prm.mass * prm.c), rho * 0., rho * pz, rho * (px + 1j * py)])
