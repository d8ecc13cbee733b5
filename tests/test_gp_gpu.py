"""GPU_Wigner2D_GPitaevskii (Strang splitting, Gross-Pitaevskii mean-field
term) on the CUDA path against golden fixtures from the reference's own class
and against the oracle (oracle/gpitaevskii.py).  Tolerance: relative 1e-10."""
import numpy as np
import pytest

from oracle.common import rel_l2
from oracle.gpitaevskii import GPitaevskiiOracle
from oracle.wigner2d import WignerParams, wigner_harmonic_oscillator
from golden_cases import GP_NAMES, gp_case, obs_close
from instances import gp_instance, wigner_obs

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.mark.parametrize('name', GP_NAMES)
def test_gp_golden(name):
    g, prm, a_gp, W0, n = gp_case(name)
    inst = gp_instance(prm, a_gp, W0, n - 1)
    assert inst.Run() == 0
    assert obs_close(wigner_obs(inst), g['obs'], TOL) < TOL
    assert rel_l2(inst.W_end[::2, ::2], g['end_dec']) < TOL
    if a_gp != 0.:
        assert np.max(np.abs(inst.ProbabilitySquare_average - g['psq']) / np.abs(g['psq'])) < TOL


def test_gp_odm_256_vs_oracle():
    """256 x 256, double well, mean-field term a_GP = -0.3, ODM damping (one
    Lindblad term, weight 1), 40 steps."""
    prm = WignerParams(256, 256, 10., 10., 0.005, potential='0.05*pow(x,4) - pow(x,2)',
                       dpotential='0.2*pow(x,3) - 2.*x', kinetic='0.5*p*p', gamma=0.02, damping='ODM',
                       fp_damping=' p*p/sqrt( p*p + 0.5 ) ', epsilon=0.5, L_material=3.)
    W0 = np.ascontiguousarray(wigner_harmonic_oscillator(prm, 0, 1., -2., 0.5))
    inst = gp_instance(prm, -0.3, W0, 39)
    assert inst.Run() == 0
    obs, W, psq = GPitaevskiiOracle(prm, -0.3).run(W0, 40)
    assert obs_close(wigner_obs(inst), obs[:, 1:], TOL) < TOL
    assert rel_l2(inst.W_end_complex, W) < TOL
    assert np.max(np.abs(inst.ProbabilitySquare_average - psq) / np.abs(psq)) < TOL
