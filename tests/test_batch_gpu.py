"""Batched FP32 form against the FP64 oracle.

The norm is renormalised in FP64 every damped step, so it matches to 1e-6
(undamped instances drift by the FP32 FFT rounding, ~1e-8 per step).
The energy carries the FP32 FFT rounding: FFT noise is spread uniformly over
the grid (relative to the state's norm) and the energy observable weights it
with H(x, p), largest at the grid edges (V ~ a x^4 up to ~1e3 at |x| = 10), so
<H> drifts by ~1e-8 of max|H| over the grid per step; the bound is
1e-8 x steps x max|H|.  The state is checked to 1e-3 relative L2."""
import numpy as np
import pytest

from oracle.common import rel_l2
from oracle.wigner2d import WignerOracle
from batch_cases import random_batch, to_instance, to_params, initial_state

pytestmark = pytest.mark.gpu


def run_batch(cases, steps, warps=0, graph=True):
    from pywignercuda_b200.batch import WignerBatch
    b = WignerBatch([to_instance(c) for c in cases], warps=warps)
    W = b.pack([initial_state(c) for c in cases])
    obs = b.run(W, steps, graph=graph)
    return b, obs, b.unpack(W)


def test_mixed_sizes_against_fp64_oracle():
    cases = random_batch([64, 128, 256, 512, 128, 256], seed=3)
    cases[1]['gamma'] = 0.        # one undamped instance (no per-step normalisation)
    steps = 120
    b, obs, Ws = run_batch(cases, steps)
    for i, c in enumerate(cases):
        ref_obs, ref_W = WignerOracle(to_params(c)).run(initial_state(c), steps)
        # norm: renormalised in FP64 every damped step; an undamped instance keeps
        # the FP32 FFT rounding (~1e-8 per step)
        nb = 1e-6 if c['gamma'] else 2e-8 * steps
        assert np.max(np.abs(obs[i, :, 0] - ref_obs[:, 0])) < nb, i
        prm = to_params(c)
        hmax = np.abs(WignerOracle(prm).tab.obs_tables[8]).max()
        assert np.max(np.abs(obs[i, :, 9] - ref_obs[:, 9])) < 1e-8 * steps * hmax, i   # energy
        assert np.max(np.abs(obs[i, :, 1] - ref_obs[:, 1])) < 1e-4, i           # <x>
        assert rel_l2(Ws[i], ref_W) < 1e-3, (i, rel_l2(Ws[i], ref_W))


def test_graph_and_tile_shapes_agree():
    cases = random_batch([128, 256, 512, 1024], seed=5)
    _, o8, W8 = run_batch(cases, 20, warps=8, graph=True)
    _, o8n, W8n = run_batch(cases, 20, warps=8, graph=False)
    _, o4, W4 = run_batch(cases, 20, warps=4, graph=True)
    for a, b in zip(W8, W8n):
        assert np.array_equal(a, b)
    # the tile width decides which two columns share a packed sequence (their FP32
    # roundings mix), so 8 and 4 warps agree to FP32 level (20 steps)
    for a, b in zip(W8, W4):
        assert np.max(np.abs(a - b)) < 1e-5 * np.max(np.abs(a))
    assert np.array_equal(o8, o8n)
    assert np.max(np.abs(o8 - o4)) < 1e-4      # the <x> bound of the FP64 comparison above


def test_autotune_and_continue():
    import torch
    from pywignercuda_b200.batch import WignerBatch
    cases = random_batch([256, 512, 1024, 128], seed=7)
    b = WignerBatch([to_instance(c) for c in cases])
    W0 = [initial_state(c) for c in cases]
    scratch = b.pack(W0)
    warps, ms = b.autotune(scratch, probe_steps=3)
    assert warps in (2, 4, 8) and ms[warps] > 0
    W = b.pack(W0)
    o1 = b.run(W, 10)
    o2 = b.run(W, 10, t_index0=10, continue_run=True)
    W2 = b.pack(W0)
    o = b.run(W2, 20)
    # the chunked run rounds W * scale to FP32 at the chunk boundary: FP32-level agreement
    assert np.max(np.abs(o[:, 10:, :] - o2)) < 1e-6
    assert torch.allclose(W, W2, rtol=0, atol=1e-6)
    del o1
