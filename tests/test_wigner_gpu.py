"""Wigner2D CUDA path (libwigner_b200.so, sm_100a) against the reference's own
outputs (golden fixtures) and the oracle.  Tolerance: relative L2 1e-10 on the
state, observable columns 1e-10 of their scale (see golden_cases.obs_close)."""
import numpy as np
import pytest

from oracle.common import rel_l2
from oracle.wigner2d import (WignerParams, WignerOracle, wigner_harmonic_oscillator,
                             wigner_cat_state)
from golden_cases import WIGNER_NAMES, wigner_case, obs_close
from instances import wigner_instance, wigner_obs

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.mark.parametrize('name', WIGNER_NAMES)
def test_golden(name):
    g, prm, W0, steps = wigner_case(name)
    inst = wigner_instance(prm, W0, steps)
    assert inst.Run() == 0
    assert obs_close(wigner_obs(inst), g['obs'], TOL) < TOL
    assert rel_l2(inst.W_end[::2, ::2], g['end_dec']) < TOL
    assert np.allclose([inst.W_end.sum(), (inst.W_end ** 2).sum()], g['end_sums'], rtol=1e-10, atol=1e-14)


def test_harmonic_oscillator_256_plain_1000_steps():
    """256x256, x,p in [-10,10), V = x^2/2, coherent state at (2, 0), dt = 0.01,
    1000 steps in the reference loop convention (1001 propagations)."""
    prm = WignerParams(256, 256, 10., 10., 0.01, potential='0.5*pow(x,2)', dpotential='x', gamma=0.)
    W0 = wigner_harmonic_oscillator(prm, 0, 1., 2., 0.)
    inst = wigner_instance(prm, W0, 1000)
    inst.Run()
    obs, W = WignerOracle(prm).run(W0, 1001)
    assert rel_l2(inst.W_end_complex, W) < TOL
    assert obs_close(wigner_obs(inst), obs[:1001, 1:], TOL) < TOL
    assert np.max(np.abs(inst.Norm_average - obs[:1001, 0])) < 1e-12
    # the reference's Lie (first-order) splitting keeps <H> of the coherent state within O(dt)
    assert np.max(np.abs(inst.Hamiltonian_average - inst.Hamiltonian_average[0])) < 2 * prm.dt


def test_double_well_1024_caldeira_leggett_vs_oracle():
    """1024x1024, [-12,12), V = 0.05x^4 - x^2, CL gamma = 0.1, D_theta = 0.1, f = |p|,
    cat state at +-3 (sigma 0.7), dt = 0.005; 24 propagations against the oracle."""
    prm = WignerParams(1024, 1024, 12., 12., 0.005, potential='0.05*pow(x,4) - pow(x,2)',
                       dpotential='0.2*pow(x,3) - 2*x', gamma=0.1, d_theta=0.1,
                       damping='CaldeiraLeggett', fp_damping='fabs(p)')
    W0 = wigner_cat_state(prm, 3.0, 0.7)
    inst = wigner_instance(prm, W0, 23)
    inst.Run()
    obs, W = WignerOracle(prm).run(W0, 24)
    assert rel_l2(inst.W_end_complex, W) < TOL
    assert obs_close(wigner_obs(inst), obs[:24, 1:], TOL) < TOL
    assert np.max(np.abs(inst.Norm_average - 1.)) < 1e-12


def test_exact_constants_mode_and_chunked_frames():
    prm = WignerParams(128, 64, 8., 6., 0.02, hbar=0.8, mass=1.7, potential='0.3*pow(x,2) + 0.1*cos(t)*x',
                       dpotential='0.6*x + 0.1*cos(t)', gamma=0.05, d_theta=0.01, d_lambda=0.002,
                       damping='CaldeiraLeggett', fp_damping=' p*p/sqrt( p*p + 0.5 ) ', constants='exact')
    W0 = wigner_harmonic_oscillator(prm, 0, 1., 1., -0.5)
    inst = wigner_instance(prm, W0, 60, skip_frames=7, exact=True)
    inst.Run()
    obs, W = WignerOracle(prm).run(W0, 61)
    assert rel_l2(inst.W_end_complex, W) < TOL
    assert obs_close(wigner_obs(inst), obs[:61, 1:], TOL) < TOL
    assert sorted(inst.frames) == list(range(0, 61, 7))


def test_bad_inputs_raise():
    from pywignercuda_b200 import WignerArgumentError, WignerCompileError
    prm = WignerParams(96, 64, 8., 6., 0.02)
    with pytest.raises(WignerArgumentError):
        wigner_instance(prm, np.zeros((64, 96)), 5)
    prm = WignerParams(64, 64, 8., 6., 0.02, potential='0.5*pow(x,2) + float64(0.)')  # numpy-only name
    with pytest.raises(WignerCompileError):
        wigner_instance(prm, np.zeros((64, 64)), 5)


def test_odm_1024_vs_oracle():
    """ODM Lindblad damping at 1024x1024 (the reference's ODM notebook physics:
    V = x^2/2, gamma = 0.07/4, L = 3, f = p^2/sqrt(p^2 + 0.5)), 6 propagations."""
    prm = WignerParams(1024, 1024, 12., 12., 0.005, potential='0.5*pow(x,2)', dpotential='x',
                       gamma=0.07 / 4., damping='ODM', fp_damping=' p*p/sqrt( p*p + 0.5 ) ',
                       epsilon=0.5, L_material=3.)
    W0 = wigner_harmonic_oscillator(prm, 0, 1., 0., 3.)
    inst = wigner_instance(prm, W0, 5)
    inst.Run()
    obs, W = WignerOracle(prm).run(W0, 6)
    assert rel_l2(inst.W_end_complex, W) < TOL
    assert obs_close(wigner_obs(inst), obs[:6, 1:], TOL) < TOL


def test_odm_samples_of_the_complex_normalised_state():
    """ODM damping on a time-dependent double well with both diffusions, 64 x 32.
    The first-order Lindblad term does not keep sum W real, so the normalisation
    factor s has a phase and each sample is Re(s Z) = s.x Re Z - s.y Im Z of the
    moment sums Z; without the s.y term the samples here were off by ~7e-9 of
    their scale.  The negative area differs from the reference by construction:
    the kernels pick the points by the sign of Re W of the un-normalised state
    and scale the sum by s afterwards, while the reference picks them by the
    sign of Re(s W) of the normalised state.  With s = s.x + i s.y the two
    selections differ only at points where |Re W| < |s.y / s.x| |Im W|; the
    difference is bounded by |s| times the sum of |W| over those points, which
    for this case (|s.y / s.x| of order gamma dt, Im W at rounding level on the
    small points) is below 1e-12, the absolute bar here."""
    prm = WignerParams(64, 32, 10., 8., 0.01, d_theta=0.1, d_lambda=0.05, gamma=0.1,
                       potential='0.05*pow(x,4) - pow(x,2) + 0.2*x*sin(3.*t)',
                       dpotential='0.2*pow(x,3) - 2.*x + 0.2*sin(3.*t)', damping='ODM', fp_damping='fabs(p)',
                       L_material=1.)
    X = np.fft.fftshift(np.linspace(-10., 10. - 20. / 64, 64))[np.newaxis, :]
    P = np.fft.fftshift(np.linspace(-8., 8. - 16. / 32, 32))[:, np.newaxis]
    W0 = np.ascontiguousarray(np.exp(-(X - 1.5) ** 2 - (P + 0.5) ** 2 * 1.3) + 0. * 1j)
    inst = wigner_instance(prm, W0, 3)
    assert inst.Run() == 0
    obs, W = WignerOracle(prm).run(W0, 4)
    assert rel_l2(inst.W_end_complex, W) < TOL
    got = wigner_obs(inst)
    assert obs_close(got[:, :9], obs[:4, 1:10], TOL) < TOL
    assert np.max(np.abs(got[:, 9] - obs[:4, 10])) < 1e-12


@pytest.mark.parametrize('tma', ['1', '0'])
def test_register_fft_passes_opt_in(monkeypatch, tma):
    """The opt-in register-FFT x- and p-pass (WIG_RF=1), with the p-pass tile loaded by
    2-D tensor copies (WIG_TMA unset) or by thread loads (WIG_TMA=0): the 256^2 harmonic
    oscillator (1001 propagations) and the 1024^2 Caldeira-Leggett double well (24)
    against the oracle at the parity bar."""
    monkeypatch.setenv('WIG_RF', '1')
    monkeypatch.setenv('WIG_TMA', tma)
    prm = WignerParams(256, 256, 10., 10., 0.01, potential='0.5*pow(x,2)', dpotential='x', gamma=0.)
    W0 = wigner_harmonic_oscillator(prm, 0, 1., 2., 0.)
    inst = wigner_instance(prm, W0, 1000)
    inst.Run()
    obs, W = WignerOracle(prm).run(W0, 1001)
    assert rel_l2(inst.W_end_complex, W) < TOL
    assert obs_close(wigner_obs(inst), obs[:1001, 1:], TOL) < TOL
    prm = WignerParams(1024, 1024, 12., 12., 0.005, potential='0.05*pow(x,4) - pow(x,2)',
                       dpotential='0.2*pow(x,3) - 2*x', gamma=0.1, d_theta=0.1,
                       damping='CaldeiraLeggett', fp_damping='fabs(p)')
    W0 = wigner_cat_state(prm, 3.0, 0.7)
    inst = wigner_instance(prm, W0, 23)
    inst.Run()
    obs, W = WignerOracle(prm).run(W0, 24)
    assert rel_l2(inst.W_end_complex, W) < TOL
    assert obs_close(wigner_obs(inst), obs[:24, 1:], TOL) < TOL
