"""Generate the golden fixtures in this directory from the reference's own code.

Runs ``GPU_Wigner2D_FFT`` / ``GPU_Wigner2D_ODM2`` / ``GPU_FokkerPlank2D_FFT`` /
``GPU_Wigner2D_GPitaevskii`` / ``GPU_Wigner2D_GPitaevskii_Bloch`` / ``GPU_Dirac2D`` / ``GPU_Dirac3D`` from the
reference checkout through ``oracle.ref_harness`` (the reference's Python-2
host code and its CUDA-C kernel strings, compiled for the CPU; ``numpy.fft``
standing in for cuFFT) and stores, per case:

* ``params``  -- JSON of the constructor arguments / instance attributes;
* ``obs``     -- the per-step arrays ``Run()`` leaves on the instance, in the
  reference's column order (Wigner: X, X2, P, P2, XP, dPotentialdX,
  PdPotentialdX, XdPotentialdX, Hamiltonian, negativeArea; Dirac: X, Y,
  Alpha1, Alpha2, Beta, KEnergy, Potential_0; Dirac3D: X, Y, Z, Alpha1, Alpha2,
  Alpha3, Potential_0, Px, Py, Pz, K_Energy);
* ``end_dec`` -- the final state (``W_end`` or ``Psi_end``) decimated by 2 in
  each grid axis (Dirac3D: by 4 in z) to keep the files small, and ``end_sums`` -- full-grid sums
  (sum, sum of squares of the real part; for Dirac per component sum |psi|^2).

Initial states are built by the oracle's initial-state helpers (the same
arrays are fed to the reference run); ``init_sum`` records their checksum.

The reference GPU class needs X_gridDIM to be a multiple of 512 (its kernels
launch X/512 blocks of 512 threads), so Wigner cases use 512 x-points.

Usage:  PYWIGNER_REFERENCE=<reference checkout> PYTHONPATH=. python tests/golden/make_golden.py [case ...]
The environment variable names the reference checkout; the tests only read
the .npz files this script writes.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref_harness as h                       # noqa: E402
from oracle.wigner2d import (WignerParams, wigner_harmonic_oscillator,  # noqa: E402
                             wigner_cat_state)
from oracle.dirac2d import DiracParams, spinor_particle_spin_up       # noqa: E402
from oracle.dirac3d import Dirac3DParams, spinor_particle_spin_up_3d  # noqa: E402

WIGNER_CASES = {
    # harmonic oscillator, no damping (the physics of the 256^2 plain case)
    'wigner_ho_plain': dict(n_x=512, n_p=128, x_amplitude=10., p_amplitude=10., dt=0.01,
                            potential='0.5*pow(x,2)', dpotential='x', gamma=0.,
                            damping='CaldeiraLeggett', fp_damping='fabs(p)',
                            time_steps=1000, init=('ho', 0, 1., 2., 0.)),
    # double well + Caldeira-Leggett (the physics of the 1024^2 case, smaller grid)
    'wigner_cl_doublewell': dict(n_x=512, n_p=256, x_amplitude=12., p_amplitude=12., dt=0.005,
                                 potential='0.05*pow(x,4) - pow(x,2)',
                                 dpotential='0.2*pow(x,3) - 2*x', gamma=0.1, d_theta=0.1,
                                 damping='CaldeiraLeggett', fp_damping='fabs(p)',
                                 time_steps=300, init=('cat', 3., 0.7)),
    # time-dependent potential, D_Lambda, smooth CL damping function, hbar != 1
    'wigner_cl_timedep': dict(n_x=512, n_p=128, x_amplitude=10., p_amplitude=8., dt=0.01,
                              hbar=0.7, mass=1.3, d_theta=0.02, d_lambda=0.001,
                              potential='0.5*pow(x,2) + 0.3*sin(2.*t)*x',
                              dpotential='x + 0.3*sin(2.*t)', gamma=0.05,
                              damping='CaldeiraLeggett', fp_damping=' p*p/sqrt( p*p + 0.5 ) ',
                              time_steps=100, init=('ho', 0, 1., -1., 0.5)),
    # ODM Lindblad damping
    'wigner_odm': dict(n_x=512, n_p=128, x_amplitude=12., p_amplitude=12., dt=0.005,
                       potential='0.5*pow(x,2)', dpotential='x', gamma=0.07 / 4.,
                       damping='ODM', fp_damping=' p*p/sqrt( p*p + 0.5 ) ',
                       epsilon=0.5, L_material=3., time_steps=100, init=('ho', 0, 1., 0., 3.)),
    # GPU_Wigner2D_ODM2: kinetic from the string, damping + pumping terms
    'wigner_odm2': dict(n_x=512, n_p=128, x_amplitude=12., p_amplitude=12., dt=0.005,
                        potential='0.5*pow(x,2)', dpotential='x', kinetic='0.5*p*p/1.0',
                        gamma=0.07 / 4., damping='ODM', fp_damping=' p*p/sqrt( p*p + 0.5 ) ',
                        epsilon=0.5, L_material=3., odm2=True, weight1=1.0, weight2=0.5,
                        time_steps=60, init=('ho', 0, 1., 0., 3.)),
    # GPU_FokkerPlank2D_FFT: classical (KvN) potential factor from the dPotential string,
    # time-dependent force, Caldeira-Leggett, normalisation 'Wigner'
    'fokkerplanck_kvn': dict(n_x=512, n_p=128, x_amplitude=10., p_amplitude=10., dt=0.005,
                             potential='0.05*pow(x,4) - pow(x,2) + 0.3*sin(3.*t)*x',
                             dpotential='0.2*pow(x,3) - 2.*x + 0.3*sin(3.*t)', gamma=0.05,
                             d_theta=0.05, damping='CaldeiraLeggett', fp_damping=' p*p/sqrt( p*p + 0.5 ) ',
                             kvn=True, normalization='Wigner', time_steps=100, init=('cat', 2.5, 0.7)),
    # ... with any other normalisation: damped steps are not renormalised
    'fokkerplanck_kvn_nonorm': dict(n_x=512, n_p=128, x_amplitude=10., p_amplitude=10., dt=0.01,
                                    potential='0.5*pow(x,2)', dpotential='x', gamma=0.1, d_theta=0.1,
                                    damping='CaldeiraLeggett', fp_damping='fabs(p)', kvn=True,
                                    normalization='none', time_steps=60, init=('ho', 0, 1., 2., 0.)),
}

# GPU_Wigner2D_GPitaevskii (Strang splitting, Gross-Pitaevskii term)
GP_CASES = {
    'gp_cl': dict(n_x=512, n_p=128, x_amplitude=10., p_amplitude=10., dt=0.01, potential='0.5*pow(x,2)',
                  dpotential='x', kinetic='0.5*p*p', gamma=0.05, d_theta=0.05, damping='CaldeiraLeggett',
                  fp_damping=' p*p/sqrt( p*p + 0.5 ) ', gp_coefficient=0.5, time_steps=80,
                  init=('ho', 0, 1., 1., 0.)),
    'gp_odm': dict(n_x=512, n_p=128, x_amplitude=10., p_amplitude=10., dt=0.005,
                   potential='0.05*pow(x,4) - pow(x,2)', dpotential='0.2*pow(x,3) - 2.*x', kinetic='0.5*p*p',
                   gamma=0.02, damping='ODM', fp_damping=' p*p/sqrt( p*p + 0.5 ) ', epsilon=0.5, L_material=3.,
                   gp_coefficient=-0.3, time_steps=40, init=('ho', 0, 1., -2., 0.5)),
    'gp_strang_plain': dict(n_x=512, n_p=128, x_amplitude=10., p_amplitude=10., dt=0.01,
                            potential='0.05*pow(x,4) - pow(x,2) + 0.2*sin(2.*t)*x',
                            dpotential='0.2*pow(x,3) - 2.*x + 0.2*sin(2.*t)', kinetic='0.5*p*p',
                            d_lambda=0.001, gamma=0., gp_coefficient=0., time_steps=100,
                            init=('cat', 2.5, 0.7)),
}

# GPU_Wigner2D_GPitaevskii_Bloch (imaginary time, adaptive step)
BLOCH_CASES = {
    'bloch_gp': dict(n_x=512, n_p=128, x_amplitude=10., p_amplitude=10., dt=0.02, potential='0.5*pow(x,2)',
                     dpotential='x', kinetic='0.5*p*p', gp_coefficient=1.0, time_steps=60,
                     init=('ho', 0, 1., 1., 0.5)),
    # a second case: double well with a large step -- 9 of 40 steps are rejected and dt halved
    'bloch_gp_doublewell': dict(n_x=512, n_p=128, x_amplitude=10., p_amplitude=10., dt=1.0,
                                potential='0.05*pow(x,4) - pow(x,2)', dpotential='0.2*pow(x,3) - 2.*x',
                                kinetic='0.5*p*p', gp_coefficient=0.3, time_steps=40,
                                init=('ho', 0, 1., -2.5, 0.3)),
}
# (The reference's Bloch Run needs GPitaevskiiCoeff != 0: with 0 it reads its
# marginal buffer before creating it, GPU_Wigner2D_GPitaevskii.py:2145-2176.)

DIRAC_CASES = {
    # softened Coulomb, c = 137.036 (the physics of the 512^2 case, smaller grid)
    'dirac_coulomb': dict(n_x=128, n_y=128, x_amplitude=12., y_amplitude=12., dt=1e-4,
                          mass=1., c=137.036, A0='-1./sqrt(x*x+y*y+0.5)', A1='0.', A2='0.',
                          A3='0.', time_steps=300, p_init=(5., 0.)),
    # magnetic field through A1, A2 (symmetric gauge), c = 1
    'dirac_magnetic': dict(n_x=128, n_y=128, x_amplitude=12., y_amplitude=12., dt=0.01,
                           mass=1., c=1., A0=' 0.1*x ', A1='-0.5*y', A2=' 0.5*x', A3=' 0.2 ',
                           time_steps=100, p_init=(1., 0.5)),
}

# GPU_Dirac3D on cubic grids only: its plan cufftPlanMany(3, [X, Y, Z]) matches the (Z, Y, X)
# arrays when X == Z (the harness transforms the arrays as laid out)
DIRAC3D_CASES = {
    # softened Coulomb, c = 137.036, packet moving along x and z
    'dirac3d_coulomb': dict(n_x=32, n_y=32, n_z=32, x_amplitude=8., y_amplitude=8., z_amplitude=8., dt=1e-4,
                            mass=1., c=137.036, A0='-1./sqrt(x*x+y*y+z*z+0.5)', A1='0.', A2='0.', A3='0.',
                            time_steps=20, p_init=(3., 0., 1.)),
    # vector potential (field along z plus A3), time-dependent trap, unequal amplitudes, c = 20
    'dirac3d_field': dict(n_x=32, n_y=32, n_z=32, x_amplitude=8., y_amplitude=6., z_amplitude=7., dt=2e-3,
                          mass=1., c=20., A0='0.5*(x*x+y*y+z*z)*(1.+0.1*sin(5.*t))', A1='-0.5*y', A2='0.5*x',
                          A3='0.2*z', time_steps=20, p_init=(1., -0.5, 0.5)),
}


def wigner_initial(prm, init):
    if init[0] == 'ho':
        return np.ascontiguousarray(wigner_harmonic_oscillator(prm, *init[1:]))
    return wigner_cat_state(prm, *init[1:])


def run_wigner_case(name, c):
    m = h.load_reference_module('GPU_Wigner2D_FFT')
    prm_keys = {k: v for k, v in c.items() if k not in ('time_steps', 'init')}
    prm = WignerParams(**prm_keys)
    odm2 = c.get('odm2', False)
    kvn = c.get('kvn', False)
    base = m.GPU_Wigner2D_ODM2 if odm2 else (m.GPU_FokkerPlank2D_FFT if kvn else m.GPU_Wigner2D_FFT)

    class Instance(base):
        def __init__(self):
            self.dampingFunction = prm.damping
            self.grossPitaevskiiCoefficient = 0.0
            self.fp_Damping_String = prm.fp_damping
            self.epsilon = prm.epsilon
            self.L_material = prm.L_material
            self.SetTimeTrack(prm.dt, c['time_steps'], 10 ** 9, fileName='/tmp/_golden_%s.hdf5' % name)
            if kvn:
                self.kinematicString = prm.kinetic
                base.__init__(self, prm.n_x, prm.n_p, prm.x_amplitude, prm.p_amplitude, prm.hbar,
                              prm.mass, prm.d_theta, prm.d_lambda, prm.gamma, prm.potential,
                              prm.dpotential, normalization=prm.normalization)
            elif odm2:
                base.__init__(self, prm.n_x, prm.n_p, prm.x_amplitude, prm.p_amplitude, prm.hbar,
                              prm.mass, prm.d_theta, prm.d_lambda, prm.gamma, prm.weight1,
                              prm.weight2, prm.potential, prm.dpotential, prm.kinetic)
            else:
                base.__init__(self, prm.n_x, prm.n_p, prm.x_amplitude, prm.p_amplitude, prm.hbar,
                              prm.mass, prm.d_theta, prm.d_lambda, prm.gamma, prm.potential,
                              prm.dpotential, prm.kinetic)
    W0 = wigner_initial(prm, c['init'])
    with h.quiet():
        inst = Instance()
        inst.W_init = W0.copy()
        inst.Run()
    obs = np.stack([inst.X_average, inst.X2_average, inst.P_average, inst.P2_average,
                    inst.XP_average, inst.dPotentialdX_average, inst.PdPotentialdX_average,
                    inst.XdPotentialdX_average, inst.Hamiltonian_average, inst.negativeArea], 1)
    W = np.asarray(inst.W_end.real)
    return dict(params=json.dumps(c), obs=obs, end_dec=W[::2, ::2].copy(),
                end_sums=np.array([W.sum(), (W * W).sum()]),
                init_sum=np.array([W0.sum(), (W0 * W0).sum()]))


def run_gp_case(name, c):
    m = h.load_reference_module('GPU_Wigner2D_GPitaevskii')
    prm_keys = {k: v for k, v in c.items() if k not in ('time_steps', 'init', 'gp_coefficient')}
    prm = WignerParams(**prm_keys)

    class Instance(m.GPU_Wigner2D_GPitaevskii):
        def __init__(self):
            self.dampingFunction = prm.damping
            self.GPitaevskiiCoeff = c['gp_coefficient']
            self.fp_Damping_String = prm.fp_damping
            self.epsilon = prm.epsilon
            self.L_material = prm.L_material
            self.SetTimeTrack(prm.dt, c['time_steps'], 10 ** 9, fileName='/tmp/_golden_%s.hdf5' % name)
            m.GPU_Wigner2D_GPitaevskii.__init__(self, prm.n_x, prm.n_p, prm.x_amplitude, prm.p_amplitude,
                                                prm.hbar, prm.mass, prm.d_theta, prm.d_lambda, prm.gamma,
                                                prm.potential, prm.dpotential, prm.kinetic)
    W0 = wigner_initial(prm, c['init'])
    with h.quiet():
        inst = Instance()
        inst.W_init = W0.copy()
        inst.Run()
    obs = np.stack([inst.X_average, inst.X2_average, inst.P_average, inst.P2_average,
                    inst.XP_average, inst.dPotentialdX_average, inst.PdPotentialdX_average,
                    inst.XdPotentialdX_average, inst.Hamiltonian_average, inst.negativeArea], 1)
    W = np.asarray(inst.W_end.real)
    psq = np.asarray(inst.ProbabilitySquare_average, dtype=np.float64)
    return dict(params=json.dumps(c), obs=obs, psq=psq, end_dec=W[::2, ::2].copy(),
                end_sums=np.array([W.sum(), (W * W).sum()]),
                init_sum=np.array([W0.sum(), (W0 * W0).sum()]))


def run_bloch_case(name, c):
    m = h.load_reference_module('GPU_Wigner2D_GPitaevskii')
    prm_keys = {k: v for k, v in c.items() if k not in ('time_steps', 'init', 'gp_coefficient')}
    prm = WignerParams(**prm_keys)

    class Instance(m.GPU_Wigner2D_GPitaevskii_Bloch):
        def __init__(self):
            self.GPitaevskiiCoeff = c['gp_coefficient']
            self.SetTimeTrack(prm.dt, c['time_steps'], 10 ** 9, fileName='/tmp/_golden_%s.hdf5' % name)
            m.GPU_Wigner2D_GPitaevskii_Bloch.__init__(self, prm.n_x, prm.n_p, prm.x_amplitude, prm.p_amplitude,
                                                      prm.hbar, prm.mass, prm.potential, prm.kinetic)
    W0 = wigner_initial(prm, c['init'])
    with h.quiet():
        inst = Instance()
        inst.W_init = W0.copy()
        inst.Run()
    avg = np.stack([inst.X_average, inst.X2_average, inst.P_average, inst.P2_average,
                    inst.Hamiltonian_average], 1)
    W = np.asarray(inst.W_0.real)
    nle = np.asarray(getattr(inst, 'NonLinearEnergyHistory', np.zeros(0)), dtype=np.float64)
    return dict(params=json.dumps(c), avg=avg, energy=np.asarray(inst.TotalEnergyHistory, dtype=np.float64),
                nle=nle, purity=np.asarray(inst.purity, dtype=np.float64), end_dec=W[::2, ::2].copy(),
                end_sums=np.array([W.sum(), (W * W).sum()]),
                init_sum=np.array([W0.sum(), (W0 * W0).sum()]))


def run_dirac_case(name, c):
    d = h.load_reference_module('GPU_Dirac2D')
    prm_keys = {k: v for k, v in c.items() if k not in ('time_steps', 'p_init')}
    prm = DiracParams(**prm_keys)

    class Instance(d.GPU_Dirac2D):
        def __init__(self):
            self.mass, self.c, self.hBar = prm.mass, prm.c, prm.hbar
            self.Potential_0_String, self.Potential_1_String = prm.A0, prm.A1
            self.Potential_2_String, self.Potential_3_String = prm.A2, prm.A3
            self.fileName = '/tmp/_golden_%s.hdf5' % name
            d.GPU_Dirac2D.__init__(self, (prm.n_x, prm.n_y), (prm.x_amplitude, prm.y_amplitude),
                                   prm.dt, c['time_steps'], 10 ** 9, frameSaveMode='Density')
    psi0 = spinor_particle_spin_up(prm, c['p_init'], lambda x, y: np.exp(-(x * x + y * y) / 2.))
    with h.quiet():
        inst = Instance()
        inst.Psi_init = psi0.copy()
        inst.Run()
    obs = np.stack([inst.X_average, inst.Y_average, inst.Alpha1_average, inst.Alpha2_average,
                    inst.Beta_average, inst.KEnergy_average, inst.Potential_0_average], 1)
    P = np.asarray(inst.Psi_end)
    return dict(params=json.dumps(c), obs=obs, end_dec=P[:, ::2, ::2].copy(),
                end_sums=np.array([np.sum(np.abs(p) ** 2) for p in P]),
                init_sum=np.array([np.sum(np.abs(p) ** 2) for p in psi0]))


def run_dirac3d_case(name, c):
    d = h.load_reference_module('GPU_Dirac3D')
    prm = Dirac3DParams(**{k: v for k, v in c.items() if k not in ('time_steps', 'p_init')})

    class Instance(d.GPU_Dirac3D):
        def __init__(self):
            self.mass, self.c, self.hBar = prm.mass, prm.c, prm.hbar
            self.Potential_0_String, self.Potential_1_String = prm.A0, prm.A1
            self.Potential_2_String, self.Potential_3_String = prm.A2, prm.A3
            self.fileName = '/tmp/_golden_%s.hdf5' % name
            self.Compute_Ehrenfest_P = True
            d.GPU_Dirac3D.__init__(self, (prm.n_x, prm.n_y, prm.n_z),
                                   (prm.x_amplitude, prm.y_amplitude, prm.z_amplitude),
                                   prm.dt, c['time_steps'], 10 ** 9, frameSaveMode='Density')
    psi0 = spinor_particle_spin_up_3d(prm, c['p_init'], lambda x, y, z: np.exp(-(x * x + y * y + z * z) / 2.))
    with h.quiet():
        inst = Instance()
        inst.Psi_init = psi0.copy()
        inst.Run()
    obs = np.stack([inst.X_average, inst.Y_average, inst.Z_average, inst.Alpha1_average, inst.Alpha2_average,
                    inst.Alpha3_average, inst.Potential_0_average, inst.Px_average, inst.Py_average,
                    inst.Pz_average, np.real(inst.K_Energy_average)], 1)
    P = np.asarray(inst.Psi_end)
    return dict(params=json.dumps(c), obs=obs, end_dec=P[:, ::4, ::2, ::2].copy(),
                end_sums=np.array([np.sum(np.abs(p) ** 2) for p in P]),
                init_sum=np.array([np.sum(np.abs(p) ** 2) for p in psi0]))


# initial-state helpers: Propagator_Base.Wigner_HarmonicOscillator /
# Wigner_Half_HarmonicOscillator (GPU_Wigner2D_FFT.py:715-771) and the
# GPU_Dirac2D spinors (GPU_Dirac2D.py:419-497, 503-535, 646-701)
INIT_WIGNER = dict(n_x=64, n_p=32, x_amplitude=8., p_amplitude=6., mass=1.3, hbar=0.7)
INIT_HO = ((0, 1., 1.5, -0.5), (1, 0.8, -1., 0.3), (2, 1.2, 0.5, 1.0))
INIT_HALF = ((0, 1., 0.5, 0.2), (1, 1.1, -0.5, 0.4))
INIT_DIRAC = dict(n_x=32, n_y=16, x_amplitude=10., y_amplitude=8., mass=1., c=3.0, hbar=1.)
INIT_P = (1.5, -0.5)
INIT_LANDAU = ((5.0, 0, 1.0, -0.5, 1), (5.0, 1, 0.5, 0.5, 1), (4.0, 2, -0.5, 0.0, 2))


def modulation(x, y):
    return np.exp(-((x - 0.5) ** 2 + 1.3 * (y + 0.2) ** 2) / 2.)


def run_initial_states():
    m = h.load_reference_module('GPU_Wigner2D_FFT')
    d = h.load_reference_module('GPU_Dirac2D')
    w = INIT_WIGNER
    out = {'params': json.dumps(dict(wigner=w, ho=INIT_HO, half=INIT_HALF, dirac=INIT_DIRAC, p=INIT_P,
                                     landau=INIT_LANDAU))}
    with h.quiet():
        pb = m.Propagator_Base.__new__(m.Propagator_Base)
        pb.mass, pb.hBar = w['mass'], w['hbar']
        pb.SetPhaseSpaceBox2D(w['n_x'], w['n_p'], w['x_amplitude'], w['p_amplitude'])
        for i, a in enumerate(INIT_HO):
            out['ho_%d' % i] = np.asarray(pb.Wigner_HarmonicOscillator(*a))
        for i, a in enumerate(INIT_HALF):
            out['half_%d' % i] = np.asarray(pb.Wigner_Half_HarmonicOscillator(*a))
        c = INIT_DIRAC

        class Instance(d.GPU_Dirac2D):
            def __init__(self):
                self.mass, self.c, self.hBar = c['mass'], c['c'], c['hbar']
                self.Potential_0_String = self.Potential_1_String = '0.'
                self.Potential_2_String = self.Potential_3_String = '0.'
                self.fileName = '/tmp/_golden_init.hdf5'
                d.GPU_Dirac2D.__init__(self, (c['n_x'], c['n_y']), (c['x_amplitude'], c['y_amplitude']), 1e-3, 1,
                                       10 ** 9, frameSaveMode='Density')
        inst = Instance()
        for name in ('Spinor_Particle_SpinUp', 'Spinor_Particle_SpinDown', 'Spinor_AntiParticle_SpinDown',
                     'Spinor_AntiParticle_SpinUp'):
            out[name] = np.asarray(getattr(inst, name)(INIT_P, modulation))
        for i, a in enumerate(INIT_LANDAU):
            out['landau_%d' % i] = np.asarray(inst.LandauLevelSpinor(*a))
        for sign in (1, -1):
            out['filter_%+d' % sign] = np.asarray(inst.FilterElectrons(sign, out['Spinor_Particle_SpinUp']))
    return out


def main(names):
    if 'initial_states' in names:
        path = os.path.join(HERE, 'initial_states.npz')
        np.savez_compressed(path, **run_initial_states())
        print('%-22s %7.1f KB' % ('initial_states', os.path.getsize(path) / 1e3))
        names = [n for n in names if n != 'initial_states']
        if not names:
            return
    cases = dict(WIGNER_CASES)
    cases.update(GP_CASES)
    cases.update(BLOCH_CASES)
    cases.update(DIRAC_CASES)
    cases.update(DIRAC3D_CASES)
    for name in names or list(cases):
        t0 = time.time()
        c = cases[name]
        if name in DIRAC_CASES:
            out = run_dirac_case(name, c)
        elif name in DIRAC3D_CASES:
            out = run_dirac3d_case(name, c)
        elif name in GP_CASES:
            out = run_gp_case(name, c)
        elif name in BLOCH_CASES:
            out = run_bloch_case(name, c)
        else:
            out = run_wigner_case(name, c)
        path = os.path.join(HERE, name + '.npz')
        np.savez_compressed(path, **out)
        print('%-22s %6.1fs  %7.1f KB' % (name, time.time() - t0, os.path.getsize(path) / 1e3))


if __name__ == '__main__':
    main(sys.argv[1:])
