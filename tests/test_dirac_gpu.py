"""Dirac2D CUDA path against the reference's own outputs and the oracle
(relative L2 1e-10 on the spinor, observables 1e-10 of their scale)."""
import numpy as np
import pytest

from oracle.common import rel_l2
from oracle.dirac2d import DiracParams, DiracOracle, spinor_particle_spin_up
from golden_cases import dirac_case, obs_close
from instances import dirac_instance, dirac_obs

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.mark.parametrize('name', ['dirac_coulomb', 'dirac_magnetic'])
def test_golden(name):
    g, prm, psi0, steps = dirac_case(name)
    inst = dirac_instance(prm, psi0, steps)
    assert inst.Run() == 0
    assert obs_close(dirac_obs(inst), g['obs'], TOL) < TOL
    assert rel_l2(inst.Psi_end[:, ::2, ::2], g['end_dec']) < TOL


def test_coulomb_512_vs_oracle():
    """512x512, [-12,12)^2, c = 137.036, -1/sqrt(r^2+0.5), packet p0 = (5, 0),
    sigma 1, dt = 1e-4: 40 steps against the oracle, all 10 columns."""
    prm = DiracParams(512, 512, 12., 12., 1e-4, A0='-1./sqrt(x*x+y*y+0.5)')
    psi0 = spinor_particle_spin_up(prm, (5., 0.), lambda x, y: np.exp(-(x * x + y * y) / 2.))
    inst = dirac_instance(prm, psi0, 40, skip_frames=16)
    inst.Run()
    obs, P = DiracOracle(prm).run(psi0, 40)
    assert rel_l2(inst.Psi_end, P) < TOL
    got = np.stack([dirac_obs(inst).T[k] for k in range(7)] + [inst.Px_average, inst.Py_average,
                                                               inst.NormKept_average], 1)
    # chunk starts (every 16 steps) report norm_kept = 1 by construction
    ref = obs.copy()
    ref[16::16, 9] = 1.
    assert obs_close(got, ref, TOL) < TOL
    assert sorted(inst.frames) == [0, 16, 32]     # t_index % skipFrames == 0 (GPU_Dirac2D.py:1107)
