"""Failure statuses of a run, as cufftCheckStatus turns a cuFFT status into an
exception in the reference (cufft_wrapper.py:67-75):

* non-finite (WIG_ERR_NONFINITE, WignerNonFiniteError): a NaN placed in a state
  on the host makes the step's observables non-finite, and the run call returns
  that status instead of numbers.  The NaN is ordinary data to the kernels:
  nothing faults or waits;
* timeout (WIG_ERR_TIMEOUT, WignerTimeoutError): a bounded device-side wait that
  runs out (forced by a test switch that never issues the awaited copy) records
  the status word and returns; the context stays usable."""
import numpy as np
import pytest
import torch

from oracle.wigner2d import WignerParams, wigner_harmonic_oscillator
from oracle.dirac2d import DiracParams, spinor_particle_spin_up
from instances import wigner_instance, dirac_instance
from batch_cases import random_batch, to_instance, initial_state

pytestmark = pytest.mark.gpu


def test_wigner_run_reports_nonfinite_state():
    from pywignercuda_b200._lib import WignerNonFiniteError
    prm = WignerParams(64, 64, 10., 10., 0.01, potential='0.5*pow(x,2)', dpotential='x', gamma=0.1, d_theta=0.1,
                       damping='CaldeiraLeggett', fp_damping='fabs(p)')
    W0 = wigner_harmonic_oscillator(prm, 0, 1., 1., 0.)
    inst = wigner_instance(prm, W0, 4)
    W = torch.from_numpy(np.ascontiguousarray(W0, dtype=np.complex128)).cuda()
    inst.propagate(W, 2)                                   # finite: runs
    W[5, 7] = float('nan')
    with pytest.raises(WignerNonFiniteError):
        inst.propagate(W, 2, continue_run=True)


def test_dirac_run_reports_nonfinite_state():
    from pywignercuda_b200._lib import WignerNonFiniteError
    dp = DiracParams(32, 32, 12., 12., 1e-4, A0='-1./sqrt(x*x+y*y+0.5)')
    psi0 = spinor_particle_spin_up(dp, (5., 0.), lambda x, y: np.exp(-(x * x + y * y) / 2.))
    inst = dirac_instance(dp, psi0, 4)
    psi = torch.from_numpy(np.ascontiguousarray(psi0, dtype=np.complex128)).cuda()
    inst.propagate(psi, 2)
    psi[1, 3, 4] = complex(float('inf'), 0.)
    with pytest.raises(WignerNonFiniteError):
        inst.propagate(psi, 2, t_index0=2)


@pytest.mark.parametrize('precision', ['f32', 'mixed'])
def test_batch_run_reports_nonfinite_state(precision):
    from pywignercuda_b200._lib import WignerNonFiniteError
    from pywignercuda_b200.batch import WignerBatch
    cases = random_batch([64, 128], seed=2)
    b = WignerBatch([to_instance(c) for c in cases], precision=precision)
    W = b.pack([initial_state(c) for c in cases])
    b.run(W, 2)
    W[int(b.offsets[1]) + 77] = float('nan')              # a point of the second instance
    with pytest.raises(WignerNonFiniteError):
        b.run(W, 2, continue_run=True)


@pytest.mark.parametrize('precision', ['f32', 'mixed'])
def test_batch_stalled_copy_reports_timeout(monkeypatch, precision):
    """A bounded wait that runs out: with WIG_BATCH_TEST_STALL=1 the staged x-pass
    announces its row copies to the mbarrier but never issues them (nothing is in
    flight), so every wait gives up after 4096 polls, records the status word and
    returns.  The run reports WignerTimeoutError (WIG_ERR_TIMEOUT) instead of
    numbers, and the context stays usable: a batch compiled without the switch then
    runs on the same device and matches the same run made beforehand."""
    from pywignercuda_b200._lib import WignerTimeoutError
    from pywignercuda_b200.batch import WignerBatch
    cases = random_batch([64, 128], seed=2)
    ref = WignerBatch([to_instance(c) for c in cases], precision=precision)
    Wr = ref.pack([initial_state(c) for c in cases])
    obs_ref = ref.run(Wr, 3)
    monkeypatch.setenv('WIG_BATCH_XSTAGE', '1')
    monkeypatch.setenv('WIG_BATCH_TEST_STALL', '1')
    b = WignerBatch([to_instance(c) for c in cases], precision=precision)
    W = b.pack([initial_state(c) for c in cases])
    with pytest.raises(WignerTimeoutError):
        b.run(W, 3, graph=False)
    del b
    monkeypatch.delenv('WIG_BATCH_TEST_STALL')
    monkeypatch.delenv('WIG_BATCH_XSTAGE')
    after = WignerBatch([to_instance(c) for c in cases], precision=precision)
    Wa = after.pack([initial_state(c) for c in cases])
    obs = after.run(Wa, 3)
    assert np.array_equal(obs, obs_ref)
    assert torch.equal(Wa, Wr)
