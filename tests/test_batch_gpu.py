"""Batched form (real FP32 storage; FP32 or mixed precision) against the FP64
oracle and the complex128 drop-in path.

The norm is renormalised in FP64 every damped step, so it matches to 1e-6
(an undamped instance keeps the FP32 transforms' rounding).  The energy error
comes from transform rounding: it is spread over the grid and weighted by
H(x, p), which is largest at the grid edges (V ~ a x^4 up to ~1e3 at |x| = 10).
In FP32 it grows about linearly with the steps; the mixed form runs the
kinetic and Moyal transform pairs in FP64, which leaves the FP32 storage
rounding (local to each point) and the dissipator pairs' FP32 rounding scaled
by 2 gamma dt.  Bounds: measured errors with a stated margin."""
import numpy as np
import pytest

from oracle.common import rel_l2
from oracle.wigner2d import WignerOracle
from batch_cases import config3_cases, random_batch, to_instance, to_params, initial_state

pytestmark = pytest.mark.gpu


def run_batch(cases, steps, warps=0, graph=True, precision='f32'):
    from pywignercuda_b200.batch import WignerBatch
    b = WignerBatch([to_instance(c) for c in cases], warps=warps, precision=precision)
    W = b.pack([initial_state(c) for c in cases])
    obs = b.run(W, steps, graph=graph)
    return b, obs, b.unpack(W)


def c128_run(cases, steps):
    """The complex128 drop-in path (pinned to the oracle at 1e-10) on each
    instance, exact constants: obs[count, steps + 1, 11]."""
    import torch
    from pywignercuda_b200 import GPU_Wigner2D_FFT, _lib

    class Poly(GPU_Wigner2D_FFT):
        constants_mode = _lib.CONST_EXACT

        def __init__(self, c):
            self.dampingFunction, self.grossPitaevskiiCoefficient = 'CaldeiraLeggett', 0.
            self.fp_Damping_String = 'fabs(p)'
            self.coefficients = [c['a'], c['b']]
            self.SetTimeTrack(0.005, steps, 10 ** 9, fileName='')
            GPU_Wigner2D_FFT.__init__(self, c['n'], c['n'], 10., 10., 1., 1., c['gamma'], 0., c['gamma'],
                                      'cf[0]*pow(x,4) + cf[1]*pow(x,2)', '4.*cf[0]*pow(x,3) + 2.*cf[1]*x',
                                      '0.5*p*p')
    out = []
    for c in cases:
        inst = Poly(c)
        W = torch.from_numpy(np.ascontiguousarray(initial_state(c), dtype=np.complex128)).to('cuda')
        out.append(inst.propagate(W, steps))
        del inst
    return np.array(out)


def energy_rel(obs, ref):
    """max over samples of |dE| / max_t |E|, per instance (the trajectory's energy
    scale: a double well's E can cross zero)."""
    return np.max(np.abs(obs[:, :, 9] - ref[:, :, 9]), axis=1) / np.max(np.abs(ref[:, :, 9]), axis=1)


# bounds after 40-120 steps (state rel L2 / energy |dE| / max|E|): measured FP32 energy errors
# 2.2e-4 .. 1.6e-3 (120 steps) over runs, with a margin of ~3x; mixed: below 1e-7
BOUNDS_120 = {'f32': (3e-5, 5e-3), 'mixed': (1e-6, 1e-6)}


@pytest.mark.parametrize('precision', ['f32', 'mixed'])
def test_mixed_sizes_against_fp64_oracle(precision):
    cases = random_batch([64, 128, 256, 512, 128, 256], seed=3)
    cases[1]['gamma'] = 0.        # one undamped instance (no per-step normalisation)
    steps = 120
    b, obs, Ws = run_batch(cases, steps, precision=precision)
    sb, eb = BOUNDS_120[precision]
    for i, c in enumerate(cases):
        ref_obs, ref_W = WignerOracle(to_params(c)).run(initial_state(c), steps)
        nb = 1e-6 if c['gamma'] else 2e-8 * steps
        assert np.max(np.abs(obs[i, :, 0] - ref_obs[:, 0])) < nb, i
        er = energy_rel(obs[i:i + 1], ref_obs[None])[0]
        assert er < eb, (i, er)
        assert np.max(np.abs(obs[i, :, 1] - ref_obs[:, 1])) < 1e-4, i           # <x>
        assert rel_l2(Ws[i], ref_W.real) < sb, (i, rel_l2(Ws[i], ref_W.real))


@pytest.mark.parametrize('precision', ['f32', 'mixed'])
def test_1024_instances_of_the_batch_against_oracle(precision):
    """Two 1024^2 instances and one 512^2 instance of the 64-instance batch
    (default_rng(0)) beside smaller ones, 40 steps, against the FP64 oracle."""
    allc = config3_cases()
    big = [c for c in allc if c['n'] == 1024][:2]
    cases = big + [next(c for c in allc if c['n'] == 512), next(c for c in allc if c['n'] == 128)]
    steps = 40
    _, obs, Ws = run_batch(cases, steps, precision=precision)
    sb, eb = BOUNDS_120[precision]
    for i, c in enumerate(cases):
        ref_obs, ref_W = WignerOracle(to_params(c)).run(initial_state(c), steps)
        assert np.max(np.abs(obs[i, :, 0] - ref_obs[:, 0])) < 1e-6, i
        er = energy_rel(obs[i:i + 1], ref_obs[None])[0]
        assert er < eb, (i, c['n'], er)
        assert rel_l2(Ws[i], ref_W.real) < sb, (i, c['n'], rel_l2(Ws[i], ref_W.real))


def test_mixed_batch_2000_steps_within_1e6_of_complex128():
    """The whole 64-instance batch for its 2000 steps in the mixed form against the
    complex128 drop-in path (pinned to the oracle): norm within 1e-6, energy within
    1e-6 of the trajectory's scale at every sample and of |E| at the last one.
    The last is what stochastic rounding of the FP32 stores buys: with rounding to
    nearest, the damped 128^2 instance 27 (E decaying to 0.04) ended 4.2e-6 off."""
    cases = config3_cases()
    steps = 2000
    _, obs, _ = run_batch(cases, steps, precision='mixed')
    ref = c128_run(cases, steps)
    assert np.max(np.abs(obs[:, :, 0] - ref[:, :, 0])) < 1e-6
    er = energy_rel(obs, ref)
    assert np.max(er) < 1e-6, (np.argmax(er), np.max(er))
    ef = np.abs(obs[:, -1, 9] - ref[:, -1, 9]) / np.abs(ref[:, -1, 9])
    assert np.max(ef) < 1e-6, (np.argmax(ef), np.max(ef))


@pytest.mark.parametrize('precision', ['f32', 'mixed'])
def test_graph_and_tile_shapes_agree(precision):
    """A graph replay equals the same run launched one kernel at a time, bit for
    bit (the mixed form's stochastic rounding draws its words from the step index,
    not from launch order); 8- and 4-warp tiles agree to FP32 level."""
    cases = random_batch([128, 256, 512, 1024], seed=5)
    _, o8, W8 = run_batch(cases, 20, warps=8, graph=True, precision=precision)
    _, o8n, W8n = run_batch(cases, 20, warps=8, graph=False, precision=precision)
    _, o4, W4 = run_batch(cases, 20, warps=4, graph=True, precision=precision)
    for a, b in zip(W8, W8n):
        assert np.array_equal(a, b)
    # the tile width decides which two columns share a packed sequence (their FP32
    # roundings mix), so 8 and 4 warps agree to FP32 level (20 steps)
    for a, b in zip(W8, W4):
        assert np.max(np.abs(a - b)) < 1e-5 * np.max(np.abs(a))
    assert np.array_equal(o8, o8n)
    assert np.max(np.abs(o8 - o4)) < 1e-4      # the <x> bound of the FP64 comparison above


@pytest.mark.parametrize('precision,bound', [('f32', 1e-4), ('mixed', 1e-5)])
def test_autotune_and_continue(precision, bound):
    import torch
    from pywignercuda_b200.batch import WignerBatch
    cases = random_batch([256, 512, 1024, 128], seed=7)
    b = WignerBatch([to_instance(c) for c in cases], precision=precision)
    W0 = [initial_state(c) for c in cases]
    scratch = b.pack(W0)
    warps, ms = b.autotune(scratch, probe_steps=3)
    assert warps in (2, 4, 8) and ms[warps] > 0
    W = b.pack(W0)
    o1 = b.run(W, 10)
    o2 = b.run(W, 10, t_index0=10, continue_run=True)
    W2 = b.pack(W0)
    o = b.run(W2, 20)
    # the chunked run rounds W * scale to FP32 at the chunk boundary, and the FP32 transforms
    # carry that rounding on: FP32-level agreement, relative to each observable's scale
    # (FP32 measured 5e-5, the energy column); the mixed form's continued run draws the
    # same rounding words as the single run (t_index0 = 10), so only the boundary differs
    scale = np.maximum(np.max(np.abs(o[:, 10:, :]), axis=1, keepdims=True), 1e-3)
    assert np.max(np.abs(o[:, 10:, :] - o2) / scale) < bound
    assert torch.max(torch.abs(W - W2)).item() < 1e-5 * torch.max(torch.abs(W2)).item()
    del o1
