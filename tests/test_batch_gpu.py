"""Batched FP32 form against the FP64 oracle: norm and energy within 1e-6
(absolute, for normalised W of unit norm), state within 1e-4 relative L2."""
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
        assert np.max(np.abs(obs[i, :, 0] - ref_obs[:, 0])) < 1e-6, i           # norm
        assert np.max(np.abs(obs[i, :, 9] - ref_obs[:, 9])) < 1e-6 * max(1., np.abs(ref_obs[:, 9]).max()), i
        assert np.max(np.abs(obs[i, :, 1] - ref_obs[:, 1])) < 1e-5, i           # <x>
        assert rel_l2(Ws[i], ref_W) < 1e-4, (i, rel_l2(Ws[i], ref_W))


def test_graph_and_tile_shapes_agree():
    cases = random_batch([128, 256, 512, 1024], seed=5)
    _, o8, W8 = run_batch(cases, 20, warps=8, graph=True)
    _, o8n, W8n = run_batch(cases, 20, warps=8, graph=False)
    _, o4, W4 = run_batch(cases, 20, warps=4, graph=True)
    for a, b in zip(W8, W8n):
        assert np.array_equal(a, b)
    for a, b in zip(W8, W4):
        assert np.array_equal(a, b)            # the per-sequence math does not depend on the tile
    assert np.array_equal(o8, o8n)
    assert np.max(np.abs(o8 - o4)) < 1e-12      # reduction order only


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
    assert np.max(np.abs(o[:, 10:, :] - o2)) < 1e-9
    assert torch.allclose(W, W2, rtol=0, atol=1e-6)
    del o1
