"""Frames and output files written by Run() through the asynchronous frame
writer (pywignercuda_b200/frames.py): every frame against the oracle state of
its step, the file read back through the reference's loaders, and runs with
frames against runs without.  Tolerance: relative 1e-10 (float32 densities:
1e-6)."""
import numpy as np
import pytest

from oracle.common import rel_l2
from oracle.dirac2d import DiracOracle, DiracParams, spinor_particle_spin_up
from oracle.gpitaevskii import GPitaevskiiOracle
from oracle.wigner2d import WignerOracle, WignerParams, wigner_harmonic_oscillator
from golden_cases import obs_close
from instances import bloch_instance, dirac_instance, gp_instance, wigner_instance, wigner_obs
from pywignercuda_b200 import frames

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _cl_256():
    return WignerParams(256, 256, 10., 10., 0.01, potential='0.05*pow(x,4) - pow(x,2)',
                        dpotential='0.2*pow(x,3) - 2.*x', kinetic='0.5*p*p', gamma=0.05, d_theta=0.05,
                        fp_damping=' p*p/sqrt( p*p + 0.5 ) ')


def test_wigner_frames_and_file(tmp_path):
    """256^2 Caldeira-Leggett double well, 121 propagations, a frame every 40
    steps: frame t is the state before step t (save_Frame :1880-1882)."""
    prm = _cl_256()
    W0 = np.ascontiguousarray(wigner_harmonic_oscillator(prm, 0, 1., -1.5, 0.5))
    name = str(tmp_path / 'cl.hdf5')
    inst = wigner_instance(prm, W0, 120, skip_frames=40, file_name=name)
    assert inst.Run() == 0
    assert sorted(inst.frames) == [0, 40, 80, 120] and inst.timeRangeIndexSaved == [0, 40, 80, 120]
    o = WignerOracle(prm)
    for t in (0, 40, 80, 120):
        ref = o.initial_normalise(W0) if t == 0 else o.run(W0, t)[1]
        assert rel_l2(inst.frames[t], ref) < TOL, t
        assert np.array_equal(inst.WignerFunctionFromFile(t), inst.frames[t])
    plain = wigner_instance(prm, W0, 120)                 # no frames, no file
    assert plain.Run() == 0
    assert obs_close(wigner_obs(inst), wigner_obs(plain), 1e-13) < 1e-13
    got = wigner_obs(inst)
    inst.LoadEhrenfestFromFile()
    assert np.array_equal(wigner_obs(inst)[:, :9], got[:, :9])
    assert np.array_equal(inst.W_end, plain.W_end_complex.real) or rel_l2(inst.W_end, plain.W_end) < 1e-13
    assert np.array_equal(frames.read(name, 'negativeArea'), got[:, 9])


def test_gp_frames_follow_the_step(tmp_path):
    """256^2 mean-field term + CL, 31 steps in chunks of 10: frames follow step
    tIndex for tIndex % skipFrames == 0 (:1996-1999); the chunked run equals the
    oracle step by step, ProbabilitySquare_average included."""
    prm = _cl_256()
    W0 = np.ascontiguousarray(wigner_harmonic_oscillator(prm, 0, 1., -1.5, 0.5))
    name = str(tmp_path / 'gp.hdf5')
    inst = gp_instance(prm, 0.4, W0, 30, skip_frames=10, file_name=name)
    assert inst.Run() == 0
    assert sorted(inst.frames) == [0, 10, 20, 30]
    orc = GPitaevskiiOracle(prm, 0.4)
    obs, W, psq = orc.run(W0, 31)
    assert obs_close(wigner_obs(inst), obs[:, 1:], TOL) < TOL
    assert np.max(np.abs(inst.ProbabilitySquare_average - psq) / np.abs(psq)) < TOL
    for t in (0, 10, 20):
        assert rel_l2(inst.frames[t], orc.run(W0, t + 1)[1]) < TOL, t
    assert rel_l2(inst.frames[30], W) < TOL
    assert np.array_equal(frames.read(name, '/Ehrenfest/ProbabilitySquare_average'), inst.ProbabilitySquare_average)


@pytest.mark.parametrize('mode', ['Density', 'Spinor'])
def test_dirac_frames_and_file(tmp_path, mode):
    """256^2 Coulomb packet, 12 steps, a frame every 4 steps (after step t)."""
    prm = DiracParams(256, 256, 12., 12., 1e-4, A0='-1./sqrt(x*x+y*y+0.5)')
    psi0 = spinor_particle_spin_up(prm, (5., 0.), lambda x, y: np.exp(-(x * x + y * y) / 2.))
    name = str(tmp_path / 'dirac.hdf5')
    inst = dirac_instance(prm, psi0, 12, skip_frames=4, file_name=name, mode=mode)
    assert inst.Run() == 0
    assert sorted(inst.frames) == [0, 4, 8, 12]
    orc = DiracOracle(prm)
    for t in (4, 8, 12):
        P = orc.run(psi0, t)[1]
        if mode == 'Spinor':
            assert rel_l2(inst.frames[t], P) < TOL
            assert np.array_equal(inst.load_Spinor(t), inst.frames[t])
        else:
            ref = frames.dirac_density(P)
            assert np.max(np.abs(inst.frames[t] - ref)) < 1e-6 * np.max(ref)
            assert np.array_equal(inst.load_Density(t), inst.frames[t])
    assert str(frames.read(name, 'Potential_0_String')) == prm.A0


def test_bloch_file(tmp_path):
    """Run writes W_0 and the averages; Run_ExitedState1 adds W_1 (:2532)."""
    prm = WignerParams(128, 128, 10., 6., 0.5, potential='0.02*pow(x,4) - pow(x,2) + 0.1*x',
                       dpotential='0.08*pow(x,3) - 2.*x + 0.1', kinetic='0.5*p*p')
    W0 = np.ascontiguousarray(wigner_harmonic_oscillator(prm, 0, 1., -5., 0.3))
    name = str(tmp_path / 'bloch.hdf5')
    inst = bloch_instance(prm, 0.2, W0, 5, file_name=name)
    assert inst.Run() == 0
    assert np.array_equal(frames.read(name, 'W_0'), inst.W_0)
    assert np.array_equal(frames.read(name, '/Ehrenfest/X_Ehrenfest'), inst.X_average)
    inst.W_init = np.ascontiguousarray(wigner_harmonic_oscillator(prm, 0, 1., 5., 0.))
    assert inst.Run_ExitedState1() == 0
    assert np.array_equal(frames.read(name, 'W_1'), inst.W_1)
    assert np.array_equal(frames.read(name, 'W_0'), inst.W_0)
