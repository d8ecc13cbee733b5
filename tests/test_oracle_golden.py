"""The CPU oracle against the reference's own outputs (no GPU).

* the notebook's recorded known answer (``CPU_GPU_Wigner2D.ipynb:557,577``);
* golden fixtures produced by running the reference's own code
  (``tests/golden/make_golden.py``).
Tolerances: relative L2 1e-10 on the final state, observable columns to 1e-10
of the column's scale (the parity bar for the complex128 path).
"""
import numpy as np
import pytest

from oracle.common import rel_l2
from oracle.strang_notebook import StrangNotebook, KNOWN_MIN_W, KNOWN_NORM
from oracle.wigner2d import WignerOracle
from oracle.dirac2d import DiracOracle
from golden_cases import (WIGNER_NAMES, DIRAC_NAMES, DIRAC3D_NAMES, GP_NAMES, BLOCH_NAMES, wigner_case,
                          dirac_case, dirac3d_case, gp_case, bloch_case, obs_close)

TOL = 1e-10


def test_notebook_known_answer():
    s = StrangNotebook()
    W = s.run(s.initial_state(), 500)
    assert abs(np.min(W) - KNOWN_MIN_W) <= 1e-10 * abs(KNOWN_MIN_W)
    assert abs(np.sum(W) * s.dX * s.dP - KNOWN_NORM) <= 1e-12


@pytest.mark.parametrize('name', WIGNER_NAMES)
def test_wigner_oracle_matches_reference(name):
    g, prm, W0, steps = wigner_case(name)
    assert np.allclose([W0.sum(), (W0 * W0).sum()], g['init_sum'], rtol=1e-14, atol=0)
    o = WignerOracle(prm)
    obs, W = o.run(W0, steps + 1)
    assert obs_close(obs[:steps + 1, 1:], g['obs'], TOL) < TOL
    assert rel_l2(W.real[::2, ::2], g['end_dec']) < TOL
    Wr = W.real
    assert np.allclose([Wr.sum(), (Wr * Wr).sum()], g['end_sums'], rtol=1e-10, atol=1e-14)


@pytest.mark.parametrize('name', DIRAC_NAMES)
def test_dirac_oracle_matches_reference(name):
    g, prm, psi0, steps = dirac_case(name)
    assert np.allclose([np.sum(np.abs(p) ** 2) for p in psi0], g['init_sum'], rtol=1e-14)
    obs, P = DiracOracle(prm).run(psi0, steps)
    assert obs_close(obs[:, :7], g['obs'], TOL) < TOL
    assert rel_l2(P[:, ::2, ::2], g['end_dec']) < TOL


@pytest.mark.parametrize('name', GP_NAMES)
def test_gp_oracle_matches_reference(name):
    from oracle.gpitaevskii import GPitaevskiiOracle
    g, prm, a_gp, W0, n = gp_case(name)
    obs, W, psq = GPitaevskiiOracle(prm, a_gp).run(W0, n)
    assert obs_close(obs[:, 1:], g['obs'], 1e-12) < 1e-12
    assert rel_l2(W.real[::2, ::2], g['end_dec']) < 1e-12
    if a_gp != 0.:
        assert np.max(np.abs(psq - g['psq']) / np.abs(g['psq'])) < 1e-12


@pytest.mark.parametrize('name', BLOCH_NAMES)
def test_bloch_oracle_matches_reference(name):
    from oracle.gpitaevskii import BlochOracle
    g, prm, a_gp, W0, steps = bloch_case(name)
    # imaginary-time factors exp(-dt/4 (V + V)) span a wide range at large dt: 1e-10
    tol = 1e-10
    r = BlochOracle(prm, a_gp).run_bloch(W0, steps)
    assert obs_close(r['avg'], g['avg'], tol) < tol
    assert r['energy'].shape == g['energy'].shape            # same accepted / rejected steps
    assert np.max(np.abs(r['energy'] - g['energy'])) < tol * np.max(np.abs(g['energy']))
    assert np.max(np.abs(r['purity'] - g['purity'])) < tol
    assert np.max(np.abs(r['nle'] - g['nle'])) < tol * np.max(np.abs(g['nle']))
    assert rel_l2(r['W'].real[::2, ::2], g['end_dec']) < tol


@pytest.mark.parametrize('name', DIRAC3D_NAMES)
def test_dirac3d_oracle_matches_reference(name):
    from oracle.dirac3d import Dirac3DOracle
    g, prm, psi0, steps = dirac3d_case(name)
    assert np.allclose([np.sum(np.abs(p) ** 2) for p in psi0], g['init_sum'], rtol=1e-14)
    obs, P = Dirac3DOracle(prm).run(psi0, steps)
    assert obs_close(obs[:, :11], g['obs'], TOL) < TOL
    assert rel_l2(P[:, ::4, ::2, ::2], g['end_dec']) < TOL
    assert np.allclose([np.sum(np.abs(p) ** 2) for p in P], g['end_sums'], rtol=1e-12)
