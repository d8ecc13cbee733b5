"""Helpers to rebuild the golden cases (parameters and initial states)."""
import json
import os

import numpy as np

from oracle.wigner2d import WignerParams, wigner_harmonic_oscillator, wigner_cat_state
from oracle.dirac2d import DiracParams, spinor_particle_spin_up

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
WIGNER_NAMES = ['wigner_ho_plain', 'wigner_cl_doublewell', 'wigner_cl_timedep', 'wigner_odm',
                'wigner_odm2', 'fokkerplanck_kvn', 'fokkerplanck_kvn_nonorm']
DIRAC_NAMES = ['dirac_coulomb', 'dirac_magnetic']
DIRAC3D_NAMES = ['dirac3d_coulomb', 'dirac3d_field']


def load(name):
    z = np.load(os.path.join(GOLDEN, name + '.npz'))
    d = {k: z[k] for k in z.files}
    d['params'] = json.loads(str(d['params']))
    return d


def wigner_case(name):
    g = load(name)
    c = dict(g['params'])
    steps, init = c.pop('time_steps'), c.pop('init')
    prm = WignerParams(**c)
    if init[0] == 'ho':
        W0 = np.ascontiguousarray(wigner_harmonic_oscillator(prm, *init[1:]))
    else:
        W0 = wigner_cat_state(prm, *init[1:])
    return g, prm, W0, steps


def dirac_case(name):
    g = load(name)
    c = dict(g['params'])
    steps, p_init = c.pop('time_steps'), c.pop('p_init')
    prm = DiracParams(**c)
    psi0 = spinor_particle_spin_up(prm, tuple(p_init), lambda x, y: np.exp(-(x * x + y * y) / 2.))
    return g, prm, psi0, steps


def dirac3d_case(name):
    """(fixture, Dirac3DParams, psi0, timeSteps) of a GPU_Dirac3D case."""
    from oracle.dirac3d import Dirac3DParams, spinor_particle_spin_up_3d
    g = load(name)
    c = dict(g['params'])
    steps, p_init = c.pop('time_steps'), c.pop('p_init')
    prm = Dirac3DParams(**c)
    psi0 = spinor_particle_spin_up_3d(prm, tuple(p_init), lambda x, y, z: np.exp(-(x * x + y * y + z * z) / 2.))
    return g, prm, psi0, steps


def obs_close(got, ref, rtol):
    """Max error of each column relative to that column's largest magnitude,
    floored at 1e-3 (a column that is roundoff noise -- e.g. the negative area of
    a Gaussian state, ~1e-14 -- is compared at an absolute 1e-3 * rtol)."""
    scale = np.maximum(np.abs(ref).max(0), 1e-3)
    return float((np.abs(got - ref).max(0) / scale).max())


GP_NAMES = ['gp_cl', 'gp_odm', 'gp_strang_plain']


def gp_case(name):
    """(fixture, WignerParams, gp_coefficient, W0, iterations) of a
    GPU_Wigner2D_GPitaevskii case; Run() makes timeSteps + 1 iterations."""
    g = load(name)
    c = dict(g['params'])
    steps, init, a_gp = c.pop('time_steps'), c.pop('init'), c.pop('gp_coefficient')
    prm = WignerParams(**c)
    if init[0] == 'ho':
        W0 = np.ascontiguousarray(wigner_harmonic_oscillator(prm, *init[1:]))
    else:
        W0 = wigner_cat_state(prm, *init[1:])
    return g, prm, a_gp, W0, steps + 1


BLOCH_NAMES = ['bloch_gp', 'bloch_gp_doublewell']


def bloch_case(name):
    """(fixture, WignerParams, gp_coefficient, W0, timeSteps) of a
    GPU_Wigner2D_GPitaevskii_Bloch case."""
    g = load(name)
    c = dict(g['params'])
    steps, init, a_gp = c.pop('time_steps'), c.pop('init'), c.pop('gp_coefficient')
    prm = WignerParams(**c)
    W0 = np.ascontiguousarray(wigner_harmonic_oscillator(prm, *init[1:]))
    return g, prm, a_gp, W0, steps
