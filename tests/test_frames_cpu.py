"""File layout of the frame / observable output (pywignercuda_b200/frames.py) on
the CPU: the keys the reference writes (GPU_Wigner2D_FFT.py:844-857, :1766,
:1936-1959; GPU_Dirac2D.py:989-1006, :703-737), the .npz form used when h5py is
absent, and the loaders reading it back.  The asynchronous writer itself needs
a GPU (tests/test_frames_gpu.py)."""
import types

import numpy as np
import pytest

from pywignercuda_b200 import frames

# WriteHDF5_variables + the Hamiltonian dataset
WIGNER_HEADER = {'dx', 'dtheta', 'dp', 'dlambda', 'x_gridDIM', 'p_gridDIM', 'x_min', 'x_max', 'p_min', 'p_max',
                 'lambda_min', 'lambda_max', 'dt', 'timeSteps', 'skipFrames', 'Hamiltonian'}
# what Run writes after its loop
WIGNER_TAIL = {'timeRange', 'timeRangeIndexSaved', 'W_init', 'W_end', 'negativeArea'} | {
    'Ehrenfest/' + k for k in ('X_Ehrenfest', 'X2_Ehrenfest', 'P_Ehrenfest', 'P2_Ehrenfest', 'XP_Ehrenfest',
                               'dPotentialdX_Ehrenfest', 'PdPotentialdX_average', 'XdPotentialdX_average',
                               'Hamiltonian_average')}
DIRAC_HEADER = {'x_gridDIM', 'y_gridDIM', 'x_amplitude', 'y_amplitude', 'dx', 'dy', 'Potential_0_String',
                'Potential_1_String', 'Potential_2_String', 'Potential_3_String'}


def _wigner_stub(n=8):
    rng = np.random.default_rng(0)
    s = types.SimpleNamespace(dX=0.1, dTheta=0.2, dP=0.3, dLambda=0.4, X_gridDIM=n, P_gridDIM=n,
                              X_amplitude=1., P_amplitude=2., Lambda_range=np.linspace(-3., 2.9, n),
                              dt=0.01, timeSteps=5, skipFrames=2, Hamiltonian=rng.random((n, n)) + 0j)
    s.timeRange = np.arange(6) * 0.01
    s.timeRangeIndexSaved = [0, 2, 4]
    for _, attr in frames.EHRENFEST_KEYS:
        setattr(s, attr, rng.random(6))
    s.negativeArea = rng.random(6)
    s.W_init = rng.random((n, n)) + 1j * rng.random((n, n))
    s.W_end = rng.random((n, n))
    return s


@pytest.fixture
def no_h5py(monkeypatch):
    monkeypatch.setattr(frames, '_h5py', None)


def test_wigner_file_layout_and_loaders(tmp_path, no_h5py):
    s = _wigner_stub()
    name = str(tmp_path / 'run.hdf5')
    f = frames.open_write(name)
    frames.wigner_header(f, s)
    W2 = np.arange(64.).reshape(8, 8) * (1 + 1j)
    frames.wigner_frame(f, 2, W2)
    frames.wigner_tail(f, s)
    f.close()
    r = frames.open_read(name)
    assert set(r.keys()) == WIGNER_HEADER | WIGNER_TAIL | {'2'}
    r.close()
    assert np.array_equal(frames.read(name, '/2'), W2)
    assert frames.read(name, 'x_max') == pytest.approx(1. - 0.1)
    assert frames.read(name, 'lambda_min') == pytest.approx(-3.)
    assert np.array_equal(frames.read(name, 'Hamiltonian'), s.Hamiltonian.real)
    t = types.SimpleNamespace()
    frames.load_ehrenfest(t, name)
    for _, attr in frames.EHRENFEST_KEYS:
        assert np.array_equal(getattr(t, attr), getattr(s, attr))
    assert np.array_equal(t.W_init, s.W_init.real) and np.array_equal(t.W_end, s.W_end)
    frames.append(name, 'W_1', W2.real)                   # Run_ExitedState1 adds W_1
    assert np.array_equal(frames.read(name, 'W_1'), W2.real)
    assert np.array_equal(frames.read(name, '/2'), W2)


def test_open_write_replaces_an_old_file(tmp_path, no_h5py):
    name = str(tmp_path / 'a.hdf5')
    f = frames.open_write(name)
    f['old'] = 1
    f.close()
    f = frames.open_write(name)
    f['new'] = 2
    f.close()
    r = frames.open_read(name)
    assert r.keys() == ['new']
    r.close()
    with pytest.raises(ValueError):                      # datasets are written once, like h5py
        g = frames.open_write(name)
        g['x'] = 1
        g['x'] = 2
    with pytest.raises(FileNotFoundError):
        frames.open_read(str(tmp_path / 'missing.hdf5'))


def test_dirac_layout(tmp_path, no_h5py):
    s = types.SimpleNamespace(X_gridDIM=8, Y_gridDIM=4, X_amplitude=1., Y_amplitude=2., dX=0.25, dY=1.,
                              Potential_0_String='-1./sqrt(x*x+y*y+0.5)', Potential_1_String='0.',
                              Potential_2_String='0.', Potential_3_String='0.')
    rng = np.random.default_rng(1)
    psi = rng.random((4, 4, 8)) + 1j * rng.random((4, 4, 8))
    name = str(tmp_path / 'dirac.hdf5')
    f = frames.open_write(name)
    frames.dirac_header(f, s)
    rho = frames.dirac_frame('Density')(f, 3, psi)
    frames.dirac_frame('Spinor')(f, 5, psi)
    f.close()
    r = frames.open_read(name)
    keys = set(r.keys())
    r.close()
    spinor = {'%d/%s/5' % (k, part) for k in range(1, 5) for part in ('real', 'imag')}
    assert keys == DIRAC_HEADER | {'3'} | spinor
    ref = np.fft.fftshift(sum(np.abs(psi[k]) ** 2 for k in range(4))).astype(np.float32)
    got = frames.read(name, '/3')
    assert got.dtype == np.float32 and np.array_equal(got, ref) and np.array_equal(rho, ref)
    assert str(frames.read(name, 'Potential_0_String')) == s.Potential_0_String
    for k in range(4):
        z = frames.read(name, '%d/real/5' % (k + 1)) + 1j * frames.read(name, '%d/imag/5' % (k + 1))
        assert np.array_equal(z, psi[k])
