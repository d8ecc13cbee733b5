"""The drop-in classes' initial-state helpers against the reference's own
(tests/golden/initial_states.npz, made by tests/golden/make_golden.py from the
reference's Propagator_Base and GPU_Dirac2D methods under the CPU harness):

* Propagator_Base.Wigner_HarmonicOscillator, Wigner_Half_HarmonicOscillator
  (GPU_Wigner2D_FFT.py:715-771);
* GPU_Dirac2D.Spinor_Particle_SpinUp / SpinDown, Spinor_AntiParticle_SpinDown /
  SpinUp (GPU_Dirac2D.py:419-497), LandauLevelSpinor (:503-535) and
  FilterElectrons (:646-701).

All host code: no GPU.  The helpers evaluate the same formulas; the bar is
1e-12 relative (the reference uses scipy.fftpack and poly1d Laguerre /
Legendre polynomials, this package numpy.fft and scipy's eval_* functions)."""
import json
import os

import numpy as np
import pytest

from oracle.common import rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope='module')
def gold():
    return np.load(os.path.join(HERE, 'golden', 'initial_states.npz'))


def _wigner_base(p):
    from pywignercuda_b200.wigner2d import Propagator_Base
    pb = Propagator_Base()
    pb.mass, pb.hBar = p['mass'], p['hbar']
    pb.SetPhaseSpaceBox2D(p['n_x'], p['n_p'], p['x_amplitude'], p['p_amplitude'])
    return pb


def _dirac(p):
    from pywignercuda_b200.dirac2d import GPU_Dirac2D
    d = GPU_Dirac2D.__new__(GPU_Dirac2D)
    d.mass, d.c, d.hBar = p['mass'], p['c'], p['hbar']
    d._set_grids((p['n_x'], p['n_y']), (p['x_amplitude'], p['y_amplitude']))
    return d


def modulation(x, y):
    return np.exp(-((x - 0.5) ** 2 + 1.3 * (y + 0.2) ** 2) / 2.)


def test_wigner_harmonic_oscillator_and_half_oscillator(gold):
    prm = json.loads(str(gold['params']))
    pb = _wigner_base(prm['wigner'])
    for i, a in enumerate(prm['ho']):
        ref = gold['ho_%d' % i]
        assert rel_l2(pb.Wigner_HarmonicOscillator(*a), ref) < 1e-12, i
    for i, a in enumerate(prm['half']):
        ref = gold['half_%d' % i]
        assert rel_l2(pb.Wigner_Half_HarmonicOscillator(*a), ref) < 1e-12, i


def test_wigner_from_wavefunction(gold):
    """Wigner_FromWavefunction (this package's helper, no counterpart in the
    reference) is the half oscillator's transform for any psi: with the half
    oscillator's psi it reproduces the reference's Wigner_Half_HarmonicOscillator
    to rounding, and for psi = exp(-m (x - x0)^2 / 2 + i p0 x / hbar) it gives the
    analytic exp(-m (x - x0)^2 - (p - p0)^2 / (m hbar^2)) to the discretisation of
    the theta transform (6e-6 on the fixture's 64 x 32 grid, hbar = 0.7)."""
    prm = json.loads(str(gold['params']))
    pb = _wigner_base(prm['wigner'])
    for i, (n, omega, x0, p0) in enumerate(prm['half']):
        W = pb.Wigner_FromWavefunction(lambda X: pb.Psi_Half_HarmonicOscillator(n, omega, x0, p0, X))
        assert rel_l2(W, gold['half_%d' % i]) < 1e-12, i
    m, h, x0, p0 = pb.mass, pb.hBar, 1.5, -0.5
    W = pb.Wigner_FromWavefunction(lambda X: np.exp(-0.5 * m * (X - x0) ** 2 + 1j * p0 * X / h))
    A = np.exp(-m * (pb.X - x0) ** 2 - (pb.P - p0) ** 2 / (m * h * h))
    assert rel_l2(W, A / (A.sum() * pb.dX * pb.dP)) < 2e-5


def test_dirac_spinors_landau_levels_and_filter(gold):
    prm = json.loads(str(gold['params']))
    d = _dirac(prm['dirac'])
    p = tuple(prm['p'])
    for name in ('Spinor_Particle_SpinUp', 'Spinor_Particle_SpinDown', 'Spinor_AntiParticle_SpinDown',
                 'Spinor_AntiParticle_SpinUp'):
        assert rel_l2(getattr(d, name)(p, modulation), gold[name]) < 1e-12, name
    for i, a in enumerate(prm['landau']):
        assert rel_l2(d.LandauLevelSpinor(*a), gold['landau_%d' % i]) < 1e-12, i
    up = d.Spinor_Particle_SpinUp(p, modulation)
    for sign in (1, -1):
        assert rel_l2(d.FilterElectrons(sign, up), gold['filter_%+d' % sign]) < 1e-12, sign
