"""wig_observables_noalloc: the observable reduction for callers that cannot
allocate device memory (its scratch is a fixed device array inside the
library).  Checked through the C ABI against the observables wig_run records
for the same W, on two calls in a row (the shared scratch keeps the previous
call's contents), within the complex128 parity tolerance (1e-10 of each
observable's scale; the two reductions sum in different orders)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _instance_and_state(n_x, n_p):
    from oracle.wigner2d import WignerParams, wigner_harmonic_oscillator
    from instances import wigner_instance
    prm = WignerParams(n_x, n_p, 10., 8., 0.01, potential='0.05*pow(x,4) - 0.5*pow(x,2)',
                       dpotential='0.2*pow(x,3) - x', gamma=0.)
    W0 = wigner_harmonic_oscillator(prm, 1, 1., 1.5, -0.5)
    return wigner_instance(prm, W0, 1), W0


@pytest.mark.parametrize('n_x,n_p', [(256, 128), (1024, 512)])
def test_noalloc_matches_wig_run_twice(n_x, n_p):
    import torch
    from pywignercuda_b200 import _lib
    lib = _lib.load()
    inst, W0 = _instance_and_state(n_x, n_p)
    dev = torch.device('cuda', 0)
    W = torch.from_numpy(W0.astype(np.complex128)).to(dev)
    ref = inst.propagate(W, 0, continue_run=True)[0]          # existing entry point, no renormalisation
    tabs = [torch.from_numpy(np.array(t)).to(dev) for t in (inst._x_tab, inst._p_tab, inst._dv_tab, inst._v0_tab)]
    scale = np.maximum(np.abs(ref), 1e-3)
    for _ in range(2):
        out = torch.full((_lib.WIG_NOBS,), float('nan'), dtype=torch.float64, device=dev)
        rc = lib.wig_observables_noalloc(W.data_ptr(), n_x, n_p, inst.dX, inst.dP, float(inst.mass),
                                         *[t.data_ptr() for t in tabs], out.data_ptr(),
                                         torch.cuda.current_stream(dev).cuda_stream)
        assert rc == 0, lib.wig_last_error()
        got = out.cpu().numpy()
        assert np.all(np.abs(got - ref) <= 1e-10 * scale), (got, ref)


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    from pywignercuda_b200 import _lib
    lib = _lib.load()
    dev = torch.device('cuda', 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    p = buf.data_ptr()
    rc = lib.wig_observables_noalloc(p, 16, 8192, 0.1, 0.1, 1., p, p, p, p, p, None)
    assert rc == 1
    assert b'static scratch limit' in lib.wig_last_error()
