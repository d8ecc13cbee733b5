"""GPU_Dirac3D on the CUDA path against golden fixtures from the reference's
own class (cubic grids) and against the oracle (oracle/dirac3d.py) on a
non-cubic grid, in chunks and with frames.  Tolerance: relative 1e-10 (state:
relative L2; observables: each column within 1e-10 of its scale)."""
import numpy as np
import pytest

from oracle.common import rel_l2
from oracle.dirac3d import Dirac3DOracle, Dirac3DParams, spinor_particle_spin_up_3d
from golden_cases import DIRAC3D_NAMES, dirac3d_case, obs_close
from instances import dirac3d_instance, dirac3d_obs
from pywignercuda_b200 import frames

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _gauss(x, y, z):
    return np.exp(-(x * x + y * y + z * z) / 2.)


@pytest.mark.parametrize('name', DIRAC3D_NAMES)
def test_dirac3d_golden(name):
    g, prm, psi0, steps = dirac3d_case(name)
    inst = dirac3d_instance(prm, psi0, steps)
    assert inst.Run() == 0
    assert obs_close(dirac3d_obs(inst)[:, :11], g['obs'], TOL) < TOL
    assert rel_l2(inst.Psi_end[:, ::4, ::2, ::2], g['end_dec']) < TOL
    assert np.allclose([np.sum(np.abs(p) ** 2) for p in inst.Psi_end], g['end_sums'], rtol=1e-12)


def _field_prm():
    """64 (x) x 32 (y) x 16 (z), unequal amplitudes, vector potential and a
    time-dependent trap, c = 20."""
    return Dirac3DParams(64, 32, 16, 8., 6., 5., 2e-3, mass=1., c=20.,
                         A0='0.5*(x*x+y*y+z*z)*(1.+0.1*sin(5.*t))', A1='-0.5*y', A2='0.5*x', A3='0.2*z')


def test_dirac3d_noncubic_vs_oracle():
    prm = _field_prm()
    psi0 = spinor_particle_spin_up_3d(prm, (1., -0.5, 0.5), _gauss)
    inst = dirac3d_instance(prm, psi0, 15)
    assert inst.Run() == 0
    obs, P = Dirac3DOracle(prm).run(psi0, 15)
    assert obs_close(dirac3d_obs(inst), obs, TOL) < TOL
    assert rel_l2(inst.Psi_end, P) < TOL


def test_dirac3d_chunks_and_frames(tmp_path):
    """A frame every 4 steps splits the run into continued chunks: the result
    equals the oracle's uninterrupted run, the momentum norm of step 1 is kept
    across chunks, and each density frame is the oracle's after its step."""
    prm = _field_prm()
    psi0 = spinor_particle_spin_up_3d(prm, (1., -0.5, 0.5), _gauss)
    name = str(tmp_path / 'd3.hdf5')
    inst = dirac3d_instance(prm, psi0, 10, skip_frames=4, file_name=name)
    assert inst.Run() == 0
    orc = Dirac3DOracle(prm)
    obs, P = orc.run(psi0, 10)
    assert obs_close(dirac3d_obs(inst), obs, TOL) < TOL
    assert rel_l2(inst.Psi_end, P) < TOL
    assert sorted(inst.frames) == [0, 4, 8]
    for t in (4, 8):
        ref = frames.dirac_density(Dirac3DOracle(prm).run(psi0, t)[1])
        assert np.max(np.abs(inst.frames[t] - ref)) < 1e-6 * np.max(ref)
        assert np.array_equal(inst.load_Density(t), inst.frames[t])
    assert int(frames.read(name, 'z_gridDIM')) == 16


def test_dirac3d_spinor_slices(tmp_path):
    prm = _field_prm()
    psi0 = spinor_particle_spin_up_3d(prm, (1., -0.5, 0.5), _gauss)
    name = str(tmp_path / 'd3s.hdf5')
    inst = dirac3d_instance(prm, psi0, 6, skip_frames=3, file_name=name, mode='Spinor')
    assert inst.Run() == 0
    xy, xz = inst.load_Spinor(6)
    assert np.array_equal(xy, inst.Psi_end[:, 0]) and np.array_equal(xz, inst.Psi_end[:, :, 0])
    assert np.array_equal(inst.frames[6][0], xy)


def test_dirac3d_exact_constants_vs_oracle():
    """Exact constants (no '%f' rounding) on both sides, 32 x 16 x 32."""
    from pywignercuda_b200 import _lib
    prm = Dirac3DParams(32, 16, 32, 7.3, 5.1, 6.7, 1.7e-3, mass=1.3, c=17.3, A0='0.3*(x*x+y*y+z*z)',
                        A1='-0.4*y', A2='0.4*x', A3='0.', constants='exact')
    psi0 = spinor_particle_spin_up_3d(prm, (0.7, -0.3, 0.2), _gauss)
    inst = dirac3d_instance(prm, psi0, 8, constants_mode=_lib.CONST_EXACT)
    assert inst.Run() == 0
    obs, P = Dirac3DOracle(prm).run(psi0, 8)
    assert obs_close(dirac3d_obs(inst), obs, TOL) < TOL
    assert rel_l2(inst.Psi_end, P) < TOL


def test_dirac3d_run_host_matches_device_run():
    """dirac3_run_host (host buffers in and out) equals dirac3_run on a device tensor, bit for bit."""
    import torch
    from pywignercuda_b200 import _lib
    prm = _field_prm()
    psi0 = np.ascontiguousarray(spinor_particle_spin_up_3d(prm, (1., -0.5, 0.5), _gauss), dtype=np.complex128)
    inst = dirac3d_instance(prm, psi0, 5)
    lib = _lib.load()
    st = torch.cuda.current_stream().cuda_stream
    out = np.empty_like(psi0)
    obs_h = np.empty((5, _lib.DIRAC3_NOBS))
    _lib.check(lib.dirac3_run_host(inst._handle, psi0.ctypes.data, out.ctypes.data, 0, 5, 0, _lib.dptr(obs_h), st),
               'dirac3_run_host')
    t = torch.from_numpy(psi0.copy()).cuda()
    obs_d = inst.propagate(t, 5)
    assert np.array_equal(out, t.cpu().numpy())
    assert np.array_equal(obs_h, obs_d)
