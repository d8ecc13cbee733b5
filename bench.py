"""Benchmark: Wigner2D grid-point-steps per second on B200, FP32 batched vs
plain complex128.

Headline (value): the FP32 batched form on 64 independent instances --
square grids drawn from {128, 256, 512, 1024} with numpy default_rng(0),
V = a x^4 + b x^2 (a ~ U[0.01, 0.1], b ~ U[-1, 0.5]), Caldeira-Leggett
gamma ~ U[0, 0.2] with D_theta = 2 gamma m kT (kT = 0.5), coherent states at
x0 ~ U[-2, 2], p0 ~ U[-1, 1], amplitudes 10, dt = 0.005 -- 23.4 M grid points,
187 MB of complex64 state (larger than the 126 MB L2), all instances in one
x-pass and one p-pass launch per step, the run replayed as one CUDA graph,
tile shape from the autotuner.  One bench "step" = one propagation of every
instance.

Alongside (plain_c128): the complex128 drop-in path on the 1024x1024 double
well (V = 0.05x^4 - x^2, gamma = 0.1, D_theta = 0.1, f = |p|, cat state,
dt = 0.005), 16 replicas stepped in lock-step (256 MB > L2); the ratio of the
two is the metric's "FP32 batched vs plain complex128".  drift_vs_fp64 states
the FP32 run's norm / energy error against a complex128 run of every instance.

Other workloads: --workload c128 (the plain line alone), dirac (Dirac2D 512^2,
16 replicas), gp (GPU_Wigner2D_GPitaevskii: Strang splitting + mean-field term
on the 1024^2 double well, 16 replicas), dirac3d (GPU_Dirac3D 256^3, a 1 GB
spinor).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload batch|c128|dirac|dirac3d|gp|adjoint|shardcost]

N > 1 (torchrun): the batch has 64 N instances (N copies of the configuration's)
partitioned by cost across the ranks (weak scaling; no data-path collective, the observables are gathered to
rank 0); the replica workloads run their replicas on every rank; time = max
over ranks.  --impl reference times the oracle's CPU restatement of the reference
propagator (complex128, numpy + scipy.fft, all host cores) on a sample of the
same batch; rank 0 only.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'Wigner2D grid-pt-steps/s: FP32 batched vs plain complex128 at stated error'
UNIT = 'grid-pt-steps/s'
NX = NP = 1024
AMP = 12.
DT = 0.005
POT = '0.05*pow(x,4) - pow(x,2)'
DPOT = '0.2*pow(x,3) - 2*x'
GAMMA, D_THETA = 0.1, 0.1
REPLICAS = 16
PASS_BYTES = NX * NP * 16 * 2      # one fused pass reads and writes the c128 grid once
# dram__bytes_read.sum + dram__bytes_write.sum per p-pass launch, from the ncu captures
# summarised in profiles/wig_passes_c128_1024.md (one 1024^2 replica, whose state fits in
# L2: the capture shows one read of it, the write-back comes after the kernel) and
# profiles/wigb_passes_batch128.md (the mixed p-pass on the 128-instance batch, 46.19 M points,
# 187.04 MB read + 200.93 MB written: the state once each way plus spilled local memory; scaled
# here by points to the 64-instance batch's 23.36 M, since each pass reads and writes every point once)
NCU_TRAFFIC_PPASS = 16.94e6 + 0.005e6
NCU_TRAFFIC_BATCH = (187.04e6 + 200.93e6) * 23363584 / 46186496


def peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def cat_state(inst):
    def psi(x):
        return np.exp(-(x - 3.) ** 2 / (2 * 0.7 ** 2)) + np.exp(-(x + 3.) ** 2 / (2 * 0.7 ** 2))
    return np.ascontiguousarray(inst.Wigner_FromWavefunction(psi).real)


def make_instance(time_steps):
    from pywignercuda_b200 import GPU_Wigner2D_FFT

    class DoubleWell(GPU_Wigner2D_FFT):
        def __init__(self):
            self.dampingFunction = 'CaldeiraLeggett'
            self.grossPitaevskiiCoefficient = 0.
            self.fp_Damping_String = 'fabs(p)'
            self.SetTimeTrack(DT, time_steps, 10 ** 9, fileName='')
            GPU_Wigner2D_FFT.__init__(self, NX, NP, AMP, AMP, 1., 1., D_THETA, 0., GAMMA, POT, DPOT,
                                      '0.5*p*p')
    return DoubleWell()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.Q,
                                          '--format=csv,noheader,nounits', '-lms', '100'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in self.lines:
            f = [x.strip() for x in ln.split(',')]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[4:8]):
                if v.lower().startswith('active'):
                    reasons.add(name)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [], 'samples': 0}
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': max(mx), 'reasons': sorted(reasons),
                'samples': len(sm)}


def dist_setup():
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device('cuda', local))
    return world, rank, local


def barrier_max(world, value):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = 'cuda' if dist.get_backend() == 'nccl' else 'cpu'
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def batch_config(seed=0, count=64):
    """The 64-instance mixed-grid batch (see the module docstring)."""
    rng = np.random.default_rng(seed)
    sizes = rng.choice([128, 256, 512, 1024], size=count)
    a = rng.uniform(0.01, 0.1, count)
    b = rng.uniform(-1., 0.5, count)
    g = rng.uniform(0., 0.2, count)
    x0 = rng.uniform(-2., 2., count)
    p0 = rng.uniform(-1., 1., count)
    kT, mass = 0.5, 1.
    return [dict(n=int(sizes[i]), a=float(a[i]), b=float(b[i]), gamma=float(g[i]),
                 d_theta=float(2 * g[i] * mass * kT), x0=float(x0[i]), p0=float(p0[i]))
            for i in range(count)]


def coherent_state(n, x0, p0, amp=10.):
    """Wigner function of the coherent state at (x0, p0), omega = m = hbar = 1,
    FFT-shifted, normalised (Wigner_HarmonicOscillator with n = 0)."""
    d = 2. * amp / n
    g = np.fft.fftshift(np.linspace(-amp, amp - d, n))
    X, P = g[np.newaxis, :], g[:, np.newaxis]
    W = np.exp(-((X - x0) ** 2 + (P - p0) ** 2))
    return W / (W.sum() * d * d)


def c128_reference_obs(cases, steps, dev):
    """complex128 drop-in runs of the batch's instances (exact constants,
    coefficient slots so one module per grid size): obs[count, steps+1, 11]."""
    import torch
    from pywignercuda_b200 import GPU_Wigner2D_FFT, _lib

    class Poly(GPU_Wigner2D_FFT):
        constants_mode = _lib.CONST_EXACT

        def __init__(self, c):
            self.dampingFunction, self.grossPitaevskiiCoefficient = 'CaldeiraLeggett', 0.
            self.fp_Damping_String = 'fabs(p)'
            self.coefficients = [c['a'], c['b']]
            self.SetTimeTrack(DT, steps, 10 ** 9, fileName='')
            GPU_Wigner2D_FFT.__init__(self, c['n'], c['n'], 10., 10., 1., 1., c['d_theta'], 0., c['gamma'],
                                      'cf[0]*pow(x,4) + cf[1]*pow(x,2)', '4.*cf[0]*pow(x,3) + 2.*cf[1]*x',
                                      '0.5*p*p')
    out = []
    for c in cases:
        inst = Poly(c)
        W = torch.from_numpy(coherent_state(c['n'], c['x0'], c['p0']).astype(np.complex128)).to(dev)
        out.append(inst.propagate(W, steps))
        del inst
    return np.array(out)


def cpu_baseline_run(max_seconds=20.0, min_steps=2, max_steps=None):
    """The oracle's restatement of the reference's step (numpy + scipy.fft, all
    host cores) on one 1024^2 instance; returns (grid-pt-steps/s, steps, seconds)."""
    from oracle.wigner2d import WignerParams, WignerOracle, wigner_cat_state
    from oracle.common import WORKERS
    prm = WignerParams(NX, NP, AMP, AMP, DT, potential=POT, dpotential=DPOT, gamma=GAMMA, d_theta=D_THETA,
                       damping='CaldeiraLeggett', fp_damping='fabs(p)')
    o = WignerOracle(prm)
    W = o.initial_normalise(wigner_cat_state(prm, 3.0, 0.7))
    W = o.step(W, 0.)                       # warm-up (tables, FFT plans)
    n, t0 = 0, time.perf_counter()
    while True:
        o.observables(W)
        W = o.step(W, (n + 1) * DT)
        n += 1
        el = time.perf_counter() - t0
        if (n >= min_steps and el >= max_seconds) or (max_steps and n >= max_steps):
            break
    return NX * NP * n / el, n, el, WORKERS


def cpu_batch_sample(cases, max_seconds=15.0):
    """The oracle (complex128, numpy + scipy.fft, all cores) on a sample of the
    batch: one instance of each grid size, stepped in turn until max_seconds."""
    from oracle.wigner2d import WignerParams, WignerOracle
    from oracle.common import WORKERS
    sample = []
    for n in (128, 256, 512, 1024):
        c = next((c for c in cases if c['n'] == n), None)
        if c is None:
            continue
        prm = WignerParams(n, n, 10., 10., DT, potential='%r*pow(x,4) + %r*pow(x,2)' % (c['a'], c['b']),
                           dpotential='0.', gamma=c['gamma'], d_theta=c['d_theta'], damping='CaldeiraLeggett',
                           fp_damping='fabs(p)', constants='exact')
        o = WignerOracle(prm)
        W = o.initial_normalise(coherent_state(n, c['x0'], c['p0']))
        W = o.step(W, 0.)                   # warm-up: tables, FFT plans
        sample.append([o, W, n])
    pts, steps, t0 = 0, 0, time.perf_counter()
    while True:
        for item in sample:
            o, W, n = item
            o.observables(W)
            item[1] = o.step(W, DT)
            pts += n * n
        steps += 1
        el = time.perf_counter() - t0
        if el >= max_seconds and steps >= 2:
            break
    return pts / el, steps, el, WORKERS, '%d rounds of one step of a 128/256/512/1024 instance' % steps


def cpu_notebook_sample(steps=20, repeats=3, warmup=10):
    """The reference notebook's own CPU propagator (real W, Strang V/2-K-V/2 with
    real FFTs; ``CPU_GPU_Wigner2D.ipynb`` cells 6-10, pyFFTW restated by scipy.fft
    on all cores) in its own configuration, 512^2: warm-up, then the median of
    ``repeats`` timed runs of ``steps`` steps, as grid-pt-steps/s."""
    from oracle.strang_notebook import StrangNotebook
    from oracle.common import WORKERS
    nb = StrangNotebook()
    W = nb.run(nb.initial_state(), warmup)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        W = nb.run(W, steps)
        times.append(time.perf_counter() - t0)
    t = sorted(times)[len(times) // 2]
    return {'value': nb.n_x * nb.n_p * steps / t, 'unit': UNIT, 'cores': WORKERS, 'kind': 'port',
            'sample': 'the notebook\'s CPU Strang path (real FFTs), 512^2, median of %d x %d steps after %d '
                      'warm-up' % (repeats, steps, warmup)}


def run_reference(args, world, rank):
    if rank != 0:
        return
    cases = batch_config()
    budget = min(120.0, 2.0 * max(args.steps, 1))
    rate, n, el, cores, what = cpu_batch_sample(cases, max_seconds=budget)
    line = {'metric': METRIC, 'value': rate, 'unit': UNIT, 'n_gpus': args.gpus, 'steps': n,
            'warmup': args.warmup, 'ms_per_step': 1e3 * el / n, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'c128', 'data': 'synthetic',
            'impl': 'reference',
            'config': {'workload': 'sample of the 64-instance mixed-grid batch (default_rng(0))',
                       'form': 'CPU restatement of GPU_Wigner2D_FFT.Run (complex128, numpy + scipy.fft)'},
            'cpu_baseline': {'value': rate, 'unit': UNIT, 'cores': cores, 'kind': 'port', 'sample': what},
            'e2e': {'value': rate, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line))


def run_c128(args, world, rank, local, steps=None, emit=True):
    """The plain complex128 drop-in path on the 1024x1024 double well, R replicas."""
    import ctypes
    import torch
    from pywignercuda_b200 import _lib
    lib = _lib.load()
    steps = steps or args.steps
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    R = args.replicas
    insts = [make_instance(steps) for _ in range(R)]
    W0 = cat_state(insts[0])
    Ws = [torch.from_numpy(W0.astype(np.complex128)).to(dev) for _ in range(R)]
    stream = torch.cuda.current_stream(dev)
    hs = (ctypes.c_void_p * R)(*[i._handle.value for i in insts])
    ws = (ctypes.c_void_p * R)(*[w.data_ptr() for w in Ws])
    obs = [np.empty((steps + 1, _lib.WIG_NOBS)) for _ in range(R)]
    obs_p = (_lib._DP * R)(*[_lib.dptr(o) for o in obs])
    _lib.check(lib.wig_run_many(hs, ws, R, 0, args.warmup, 0, None, stream.cuda_stream), 'warm-up')
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        _lib.check(lib.wig_run_many(hs, ws, R, args.warmup, steps, _lib.WIG_RUN_CONTINUE, obs_p,
                                    stream.cuda_stream), 'timed')
        e1.record(stream)
        torch.cuda.synchronize()
    ms = barrier_max(world, e0.elapsed_time(e1))
    value = world * R * NX * NP * steps / (ms / 1e3)
    # per-pass device times from a separate profiled run (events around every launch)
    nprof = min(steps, 20)
    _lib.check(lib.wig_run_many(hs, ws, R, args.warmup + steps, nprof, _lib.WIG_RUN_CONTINUE | _lib.WIG_RUN_PROFILE,
                                None, stream.cuda_stream), 'profiled')
    torch.cuda.synchronize()
    x_ms = p_ms = 0.
    launches = 0
    for i in insts:
        out = (ctypes.c_double * 2)()
        cnt = ctypes.c_int64()
        _lib.check(lib.wig_profile(i._handle, out, ctypes.byref(cnt)), 'wig_profile')
        x_ms, p_ms, launches = x_ms + out[0], p_ms + out[1], launches + cnt.value
    peak, peak_kind = peaks()
    p_gbs = PASS_BYTES / (p_ms / launches / 1e3) / 1e9
    res = {'value': value, 'unit': UNIT, 'ms_per_step': ms / steps, 'steps': steps, 'replicas': R,
           'workload': 'Wigner2D 1024x1024 double well V=0.05x^4-x^2, Caldeira-Leggett gamma=0.1 D_theta=0.1 '
                       'f=|p|, cat state, dt=0.005, complex128',
           'x_pass_us': x_ms / launches * 1e3, 'p_pass_us': p_ms / launches * 1e3,
           'p_pass_hbm_frac': p_gbs / peak,
           'max_abs_norm_error': max(float(np.max(np.abs(o[:, 0] - 1.))) for o in obs),
           'clocks': clk.summary()}
    del insts
    if emit and rank == 0:
        line = {'metric': 'Wigner2D grid-pt-steps/s (plain complex128)', 'value': value, 'unit': UNIT,
                'n_gpus': world, 'steps': steps, 'warmup': args.warmup, 'ms_per_step': ms / steps,
                'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'c128',
                'data': 'synthetic', 'config': {'workload': res['workload'], 'replicas_per_gpu': R},
                'roofline': {'bound': 'hbm', 'kernel': 'wig_ppass', 'achieved': p_gbs, 'peak': peak,
                             'unit': 'GB/s', 'frac': p_gbs / peak, 'peak_kind': peak_kind,
                             'traffic': NCU_TRAFFIC_PPASS},
                'gpu_launches': R * (2 * steps + 3), 'clocks': res['clocks']}
        print(json.dumps(line))
    return res


GP_COEF = 0.5
GP_BYTES = 160   # per grid point per Strang step: 3 passes x 32 B, 2 column-sum reads x 16 B, 2 x (8 + 8) B phase


def make_gp_instance(time_steps):
    from pywignercuda_b200 import GPU_Wigner2D_GPitaevskii

    class MeanField(GPU_Wigner2D_GPitaevskii):
        def __init__(self):
            self.dampingFunction = 'CaldeiraLeggett'
            self.GPitaevskiiCoeff = GP_COEF
            self.fp_Damping_String = 'fabs(p)'
            self.SetTimeTrack(DT, time_steps, 10 ** 9, fileName='')
            GPU_Wigner2D_GPitaevskii.__init__(self, NX, NP, AMP, AMP, 1., 1., D_THETA, 0., GAMMA, POT, DPOT,
                                              '0.5*p*p')
    return MeanField()


def run_adjoint(args, world, rank, local):
    """The differentiable form on the control configuration: 512^2, V = a x^4 - b x^2
    + eps(t) x (a = 0.05, b = 1), eps piecewise constant over 50 segments of 10 steps
    (default_rng(1), N(0, 0.1)), coherent state at (-2, 0), loss dxdp sum W_T W_target
    (target centre from default_rng(2)), 500 steps, a checkpoint every 50.  One
    gradient = the checkpointed forward sweep + the backward sweep (segment
    recomputation + adjoint steps) of WignerControl.propagate, giving dL/d(W0, eps, a, b).
    Timed with CUDA events per gradient, in complex128 and complex64, undamped and
    with Caldeira-Leggett damping (gamma = 0.1, D_theta = 0.1)."""
    import torch
    from pywignercuda_b200.adjoint import WignerControl
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    n, T, K = 512, 500, 50
    eps0 = torch.tensor(np.random.default_rng(1).normal(0., 0.1, 50), dtype=torch.float64,
                        device=dev).repeat_interleave(10).contiguous()
    c = np.random.default_rng(2).uniform(-2., 2., 2)
    d = 2. * 10. / n
    target = torch.from_numpy(coherent_state(n, float(c[0]), float(c[1]))).to(dev)
    reps = max(1, min(args.steps, 5))
    out = {}
    stream = torch.cuda.current_stream(dev)
    for prec in ('c128', 'c64'):
        for gamma in (0., 0.1):
            prop = WignerControl(n, x_amplitude=10., dt=DT, v4=0.05, v2=-1., gamma=gamma, d_theta=gamma,
                                 precision=prec)
            W0 = torch.from_numpy(coherent_state(n, -2., 0.)).to(dev).to(prop.dtype)

            def gradient():
                W0r = W0.clone().requires_grad_(True)
                eps = eps0.clone().requires_grad_(True)
                coef = torch.tensor([0.05, -1.], dtype=torch.float64, device=dev, requires_grad=True)
                WT = prop.propagate(W0r, eps, coef, checkpoint=K)
                L = (WT.real.double() * target).sum() * d * d
                L.backward()
                return L
            for _ in range(max(1, min(args.warmup, 2))):
                gradient()
            torch.cuda.synchronize()
            times = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                gradient()
                e1.record(stream)
                torch.cuda.synchronize()
                times.append(e0.elapsed_time(e1))
            ms = sorted(times)[len(times) // 2]
            # a gradient advances the grid 2 T steps forward (sweep + recomputation) and T adjoint steps
            out['%s_%s' % (prec, 'damped' if gamma else 'undamped')] = {
                'ms_per_gradient': ms, 'grid_pt_steps_per_s': n * n * 3 * T / (ms / 1e3)}
            del prop
    if rank == 0:
        print(json.dumps({'workload': 'adjoint', 'metric': 'gradient of the 500-step 512^2 control problem',
                          'unit': 'ms per gradient (median of %d)' % reps, 'higher_is_better': False,
                          'n_gpus': world, 'steps': T, 'checkpoint': K, 'forms': out,
                          'note': 'grid_pt_steps_per_s counts the forward sweep, its recomputation and the '
                                  'adjoint sweep (3 T steps of the 512^2 grid)'}))


def run_gp(args, world, rank, local):
    """GPU_Wigner2D_GPitaevskii on the 1024x1024 double well: Strang splitting,
    mean-field coefficient 0.5, Caldeira-Leggett, complex128, R replicas."""
    import ctypes
    import torch
    from pywignercuda_b200 import _lib
    from oracle.gpitaevskii import GPitaevskiiOracle
    from oracle.wigner2d import WignerParams
    lib = _lib.load()
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    R, steps = args.replicas, args.steps
    insts = [make_gp_instance(steps) for _ in range(R)]
    W0 = cat_state(insts[0])
    Ws = [torch.from_numpy(W0.astype(np.complex128)).to(dev) for _ in range(R)]
    stream = torch.cuda.current_stream(dev)
    hs = (ctypes.c_void_p * R)(*[i._handle.value for i in insts])
    ws = (ctypes.c_void_p * R)(*[w.data_ptr() for w in Ws])
    _lib.check(lib.wig_run_many(hs, ws, R, 0, args.warmup, 0, None, stream.cuda_stream), 'warm-up')
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        _lib.check(lib.wig_run_many(hs, ws, R, args.warmup, steps, _lib.WIG_RUN_CONTINUE, None,
                                    stream.cuda_stream), 'timed')
        e1.record(stream)
        torch.cuda.synchronize()
    ms = barrier_max(world, e0.elapsed_time(e1))
    value = world * R * NX * NP * steps / (ms / 1e3)
    peak, peak_kind = peaks()
    achieved = GP_BYTES * NX * NP / (ms / 1e3 / (R * steps)) / 1e9
    line = {'metric': 'Wigner2D grid-pt-steps/s (Strang + Gross-Pitaevskii, complex128)', 'value': value,
            'unit': UNIT, 'n_gpus': world, 'steps': steps, 'warmup': args.warmup, 'ms_per_step': ms / steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'c128',
            'data': 'synthetic',
            'config': {'workload': 'GPU_Wigner2D_GPitaevskii 1024x1024 double well V=0.05x^4-x^2, a_GP=0.5, '
                                   'Caldeira-Leggett gamma=0.1 D_theta=0.1 f=|p|, cat state, dt=0.005',
                       'replicas_per_gpu': R, 'l2': 'per-step working set %d MB > 126 MB L2' % (R * 24)},
            'roofline': {'bound': 'hbm', 'kernel': 'Strang step (9 launches, step average)',
                         'algorithmic_bytes_per_point': GP_BYTES, 'achieved': achieved, 'peak': peak,
                         'unit': 'GB/s', 'frac': achieved / peak, 'peak_kind': peak_kind, 'traffic': None},
            'gpu_launches': R * 9 * steps, 'clocks': clk.summary()}
    if rank == 0 and args.cpu_baseline:
        prm = WignerParams(NX, NP, AMP, AMP, DT, potential=POT, dpotential=DPOT, kinetic='0.5*p*p', gamma=GAMMA,
                           d_theta=D_THETA, damping='CaldeiraLeggett', fp_damping='fabs(p)')
        orc = GPitaevskiiOracle(prm, GP_COEF)
        W = orc.initial_normalise(W0)
        t0, n = time.perf_counter(), 0
        while time.perf_counter() - t0 < 10. or n < 1:
            W, _ = orc.step_gp(W, n * DT)
            n += 1
        el = time.perf_counter() - t0
        line['cpu_baseline'] = {'value': NX * NP * n / el, 'unit': UNIT, 'cores': os.cpu_count(), 'kind': 'port',
                                'sample': '%d Strang + GP steps of one 1024^2 instance (%.1f s)' % (n, el)}
    if rank == 0:
        print(json.dumps(line))


def batch_leg(cases, states, precision, args, world, dev):
    """One precision of the batched form on `cases`: autotune, warm-up, then K
    steps each timed on the device (CUDA events around its x-pass and p-pass
    launches) with the L2 flushed before every step (the real FP32 state, 93 MB
    for the 64-instance batch, would otherwise stay in the 126 MB L2), and the
    same K steps replayed as one CUDA graph without flushing."""
    import torch
    from pywignercuda_b200.batch import WignerBatch, instance
    fixed = getattr(args, 'warps', 0)
    batch = WignerBatch([instance(c['n'], x_amplitude=10., dt=DT, gamma=c['gamma'], d_theta=c['d_theta'],
                                  v4=c['a'], v2=c['b']) for c in cases], precision=precision, warps=fixed)
    stream = torch.cuda.current_stream(dev)
    if fixed:                                     # profiling runs: one tile shape, no autotuning
        warps, tune_ms = fixed, {}
    else:
        scratch = batch.pack(states)
        warps, tune_ms = batch.autotune(scratch, probe_steps=3)
        del scratch
    K = args.steps
    W = batch.pack(states)
    batch.run(W, args.warmup)                                           # normalises
    torch.cuda.synchronize()
    barrier(world)
    batch.run(W, K, continue_run=True, graph=False, observables=False, profile=True, flush_l2=True)
    torch.cuda.synchronize()
    x_ms, p_ms, nl = batch.profile()
    ms = barrier_max(world, (x_ms + p_ms) / nl * K)
    # the K-step graph replay, no flushing (the state may stay in L2 between steps)
    batch.run(W, K, continue_run=True, observables=False)               # captures the K-step graph
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.run(W, K, continue_run=True, observables=False)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_graph = barrier_max(world, e0.elapsed_time(e1))
    return dict(batch=batch, W=W, warps=warps, tune_ms=tune_ms, ms=ms, ms_graph=ms_graph,
                x_us=x_ms / nl * 1e3, p_us=p_ms / nl * 1e3)


def drift(obs, ref, W=None, W_ref=None):
    """FP32-storage run against the complex128 drop-in path (pinned to the oracle):
    max |d norm|, energy error as max_t |dE| / max_t |E| and at the last sample as
    |dE| / |E|, and the final state's relative L2 (worst instance)."""
    de = np.max(np.abs(obs[:, :, 9] - ref[:, :, 9]), axis=1) / np.max(np.abs(ref[:, :, 9]), axis=1)
    dfin = np.abs(obs[:, -1, 9] - ref[:, -1, 9]) / np.abs(ref[:, -1, 9])
    out = {'steps': int(obs.shape[1] - 1), 'norm_max_abs': float(np.max(np.abs(obs[:, :, 0] - ref[:, :, 0]))),
           'energy_rel_max': float(np.max(de)), 'energy_rel_final': float(np.max(dfin))}
    if W is not None:
        out['state_rel_l2_final'] = float(max(np.linalg.norm(a - b.real) / np.linalg.norm(b.real)
                                               for a, b in zip(W, W_ref)))
    return out


def c128_runs(cases, states, steps, dev, amp=10., f='fabs(p)'):
    """complex128 drop-in runs (exact constants; coefficient slots, one module per
    grid size): (obs[count, steps+1, 11], final states)."""
    import torch
    from pywignercuda_b200 import GPU_Wigner2D_FFT, _lib

    class Poly(GPU_Wigner2D_FFT):
        constants_mode = _lib.CONST_EXACT

        def __init__(self, c):
            self.dampingFunction, self.grossPitaevskiiCoefficient = 'CaldeiraLeggett', 0.
            self.fp_Damping_String = f
            self.coefficients = [c['a'], c['b']]
            self.SetTimeTrack(DT, steps, 10 ** 9, fileName='')
            GPU_Wigner2D_FFT.__init__(self, c['n'], c['n'], amp, amp, 1., 1., c['d_theta'], 0., c['gamma'],
                                      'cf[0]*pow(x,4) + cf[1]*pow(x,2)', '4.*cf[0]*pow(x,3) + 2.*cf[1]*x',
                                      '0.5*p*p')
    obs, Ws = [], []
    for c, s in zip(cases, states):
        inst = Poly(c)
        W = torch.from_numpy(np.ascontiguousarray(s, dtype=np.complex128)).to(dev)
        obs.append(inst.propagate(W, steps))
        Ws.append(W.cpu().numpy())
        del inst
    return np.array(obs), Ws


def validation(cases, states, dev):
    """Norm / energy / state error of both precisions at the configurations' full
    step counts, against the complex128 drop-in path: the 64-instance batch for
    2000 steps, and the 1024^2 double well (amplitude 12, cat state, CL gamma 0.1,
    D_theta 0.1, f = |p|) for 4000 steps."""
    from pywignercuda_b200.batch import WignerBatch, instance
    out = {}
    ref3, Wr3 = c128_runs(cases, states, 2000, dev)
    c2 = dict(n=NX, a=0.05, b=-1., gamma=GAMMA, d_theta=D_THETA)
    s2 = cat_state(make_instance(1))
    ref2, Wr2 = c128_runs([c2], [s2], 4000, dev, amp=AMP)
    for prec in ('mixed', 'f32'):
        b3 = WignerBatch([instance(c['n'], x_amplitude=10., dt=DT, gamma=c['gamma'], d_theta=c['d_theta'],
                                   v4=c['a'], v2=c['b']) for c in cases], precision=prec)
        W = b3.pack(states)
        o3 = b3.run(W, 2000)
        W3 = b3.unpack(W)
        del b3, W
        b2 = WignerBatch([instance(NX, x_amplitude=AMP, dt=DT, gamma=GAMMA, d_theta=D_THETA, v4=0.05, v2=-1.)],
                         precision=prec)
        W = b2.pack([s2])
        o2 = b2.run(W, 4000)
        W2 = b2.unpack(W)
        del b2, W
        out[prec] = {'batch_2000': drift(o3, ref3, W3, Wr3), 'double_well_1024_4000': drift(o2, ref2, W2, Wr2)}
    out['reference'] = ('complex128 drop-in path (parity-pinned to the oracle), exact constants, same inputs; '
                        'energy_rel_max = max_t |dE| / max_t |E|, energy_rel_final = |dE| / |E| at the last sample')
    return out


def merge_validation(val, world):
    """Every rank validates its own share of the batch: the batch leg's errors are
    the worst over the ranks (the double-well leg is the same run on every rank).
    Returns the merged figures on every rank, so that all ranks pick the same
    headline form."""
    if world == 1 or val is None:
        return val
    import torch.distributed as dist
    vals = [None] * world
    dist.all_gather_object(vals, val)
    out = dict(vals[0])
    for prec in ('mixed', 'f32'):
        legs = dict(vals[0][prec])
        legs['batch_2000'] = {k: (max(v[prec]['batch_2000'][k] for v in vals) if k != 'steps' else
                                  vals[0][prec]['batch_2000'][k]) for k in vals[0][prec]['batch_2000']}
        out[prec] = legs
    return out


def run_batch(args, world, rank, local):
    """Headline: the batched form on the 64-instance mixed-grid batch.  With N
    ranks the batch has 64 N instances, N copies of the configuration's (N = 1 is
    the configuration itself), partitioned by cost across the ranks (weak scaling);
    each rank runs its share, the observables are gathered to rank 0.  Both
    precisions are timed; the headline is the one whose measured norm and energy
    errors at 2000 / 4000 steps are within 1e-6 (the mixed form), the other is
    reported beside it with its errors."""
    import torch
    from pywignercuda_b200.shard import gather_observables, partition
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    # weak scaling: N copies of the configuration's batch (N = 1 is the configuration itself),
    # partitioned by cost, so that every rank's work and accuracy profile stay the configuration's
    base = batch_config(count=args.instances or 64)
    cases_all = [dict(c) for _ in range(world) for c in base]
    parts = partition([dict(n_x=c['n'], n_p=c['n'], gamma=c['gamma']) for c in cases_all], world)
    cases = [cases_all[i] for i in parts[rank]]
    grand_total = sum(c['n'] * c['n'] for c in cases_all)
    states = [coherent_state(c['n'], c['x0'], c['p0']) for c in cases]
    K = args.steps
    precs = ('mixed', 'f32') if args.precision == 'both' else (args.precision,)
    with ClockSampler(local) as clk:
        legs = {p: batch_leg(cases, states, p, args, world, dev) for p in precs}
    val = merge_validation(validation(cases, states, dev) if not args.profile_only else None, world)
    head_p = precs[0]
    if val is not None:
        ok = all(v['norm_max_abs'] <= 1e-6 and v['energy_rel_max'] <= 1e-6 and v['energy_rel_final'] <= 1e-6
                 for v in val['mixed'].values() if isinstance(v, dict))
        head_p = 'mixed' if ok else 'f32'
        if head_p not in legs:
            head_p = precs[0]
    head = legs[head_p]
    value = grand_total * K / (head['ms'] / 1e3)
    if args.profile_only:
        if rank == 0:
            print(json.dumps({'metric': METRIC, 'value': value, 'unit': UNIT, 'steps': K,
                              'forms': {p: {'ms_per_step': legs[p]['ms'] / K, 'x_pass_us': legs[p]['x_us'],
                                            'p_pass_us': legs[p]['p_us'], 'warps_per_cta': legs[p]['warps']}
                                        for p in legs},
                              'note': 'profile-only run (timed section only)'}))
        return
    batch, total = head['batch'], head['batch'].total
    peak, peak_kind = peaks()
    pass_bytes = total * 4 * 2                                        # real FP32 state read + write per pass
    dom, dom_us = ('wigb_ppass', head['p_us']) if head['p_us'] >= head['x_us'] else ('wigb_xpass', head['x_us'])
    achieved = pass_bytes / (dom_us / 1e6) / 1e9
    # e2e: pinned host state in, run (one call, graph), host state and observables out, all timed
    hin = torch.from_numpy(np.concatenate([s.astype(np.float32).ravel() for s in states])).pin_memory()
    hout = torch.empty_like(hin).pin_memory()
    stream = torch.cuda.current_stream(dev)
    Wd = torch.empty(total, dtype=torch.float32, device=dev)
    Wd.copy_(hin)
    batch.run(Wd, K, observables=False)                                 # captures this run's graph
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    Wd.copy_(hin, non_blocking=True)
    obs_run = batch.run(Wd, K)
    hout.copy_(Wd, non_blocking=True)
    f1.record(stream)
    torch.cuda.synchronize()
    gather_observables(obs_run, parts, rank)                            # the only cross-rank exchange
    e2e_ms = barrier_max(world, max(f0.elapsed_time(f1), 1e3 * (time.perf_counter() - t0)))
    for leg in legs.values():
        leg.pop('batch')
        leg.pop('W')
    del batch
    c128 = run_c128(args, world, rank, local, steps=min(K, 100), emit=False)
    forms = {p: {'value': grand_total * K / (legs[p]['ms'] / 1e3), 'ms_per_step': legs[p]['ms'] / K,
                 'ms_per_step_graph_no_flush': legs[p]['ms_graph'] / K, 'warps_per_cta': legs[p]['warps'],
                 'autotune_ms': legs[p]['tune_ms'], 'x_pass_us': legs[p]['x_us'], 'p_pass_us': legs[p]['p_us'],
                 'ratio_vs_c128': grand_total * K / (legs[p]['ms'] / 1e3) / c128['value'],
                 'drift_vs_fp64': val[p] if val else None} for p in legs}
    line = {
        'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': K, 'warmup': args.warmup,
        'ms_per_step': head['ms'] / K, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f32 storage; ' + ('FP64 kinetic/Moyal transforms, FP32 dissipator transforms' if head_p == 'mixed'
                                    else 'FP32 transforms') + '; FP64 phase arguments and observables',
        'data': 'synthetic',
        'config': {'workload': '64 Wigner2D instances, square grids from {128,256,512,1024} (default_rng(0)), '
                               'V=a x^4+b x^2, Caldeira-Leggett, coherent states, dt=0.005',
                   'form': 'batched, precision %s, real FP32 state, one x-pass + one p-pass launch per step' % head_p,
                   'instances': len(cases_all), 'instances_per_rank': [len(p) for p in parts],
                   'grid_points': grand_total, 'warps_per_cta': head['warps'],
                   'parallelism': 'instances partitioned by cost across ranks, one process per GPU, '
                                  'observables gathered to rank 0 (no data-path collective)',
                   'l2': 'state %d MB < 126 MB L2: L2 flushed (a %d MB write) before every timed step, outside '
                         'the per-launch CUDA events' % (total * 4 >> 20, 2 * 126)},
        'plain_c128': c128,
        'ratio_vs_c128': value / c128['value'],
        'forms': forms,
        'drift_vs_fp64': val[head_p] if val else None,
        'flops': batch_flops(cases_all, world, head['ms'] / K, clk.summary()),
        'roofline': {'bound': 'hbm', 'kernel': dom, 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                     'frac': achieved / peak, 'peak_kind': peak_kind, 'algorithmic_bytes_per_launch': pass_bytes,
                     'algorithmic_bytes_complex64_storage': total * 8 * 2,
                     'avg_launch_us': dom_us, 'x_pass_us': head['x_us'], 'p_pass_us': head['p_us'],
                     'traffic': NCU_TRAFFIC_BATCH},
        'e2e': {'value': grand_total * K / (e2e_ms / 1e3), 'unit': UNIT,
                'h2d_bytes_per_step': grand_total * 4 / K,
                'd2h_bytes_per_step': (grand_total * 4 + len(cases_all) * (K + 1) * 11 * 8) / K,
                'note': 'one run call (graph): upload the packed states, K propagations, download states and '
                        'observables; bytes per propagation step'},
        'gpu_launches': 2 * K + 2,
        'clocks': clk.summary(),
    }
    if rank == 0 and args.cpu_baseline:
        rate, n, el, cores, what = cpu_batch_sample(cases, max_seconds=15.0)
        line['cpu_baseline'] = {'value': rate, 'unit': UNIT, 'cores': cores, 'kind': 'port',
                                'sample': what + ' (%.1f s)' % el,
                                'notebook_strang_512': cpu_notebook_sample()}
    if rank == 0:
        print(json.dumps(line))


def run_shardcost(args, world, rank, local):
    """Per-size-class cost of the batched form for the multi-GPU partition
    (pywignercuda_b200/shard.py): for each grid size and damping, a batch of one
    class holding about 32 M points, K steps with the L2 flushed before each,
    device time per grid point per step.  Rank 0 prints one JSON line."""
    import torch
    from pywignercuda_b200.batch import WignerBatch, instance
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    prec = 'mixed' if args.precision == 'both' else args.precision
    out = {}
    for n in (128, 256, 512, 1024):
        for damped in (False, True):
            count = max(1, (1 << 25) // (n * n))
            g = 0.1 if damped else 0.
            b = WignerBatch([instance(n, x_amplitude=10., dt=DT, gamma=g, d_theta=g, v4=0.05, v2=-0.5)] * count,
                            precision=prec)
            states = [coherent_state(n, 0.5, -0.2)] * count
            scratch = b.pack(states)
            b.autotune(scratch, probe_steps=2)
            W = b.pack(states)
            b.run(W, args.warmup)
            b.run(W, args.steps, continue_run=True, graph=False, observables=False, profile=True, flush_l2=True)
            torch.cuda.synchronize()
            x_ms, p_ms, nl = b.profile()
            out['%d%s' % (n, 'd' if damped else '')] = (x_ms + p_ms) / nl * 1e6 / (count * n * n)
            del b, W, scratch
    if rank == 0:
        print(json.dumps({'workload': 'shardcost', 'precision': prec, 'unit': 'ns per grid point per step',
                          'ns_per_point_step': out}))


def batch_flops(cases, world, ms_step, clocks):
    """Algorithmic FP32 flops of one batched step: 5 N log2 N per length-N transform, N transforms
    per axis pass; 2 in the x-pass, 2 for the potential and 6 for Caldeira-Leggett order 3 (when
    damped) in the p-pass.  Against the nominal FP32 rate of the SM clock seen under load
    (148 SMs x 128 lanes x 2 flops per FMA); no measured FP32 peak exists for this pool."""
    import math
    total = 0.
    for c in cases:
        n = c['n']
        ffts = 2 + 2 + (6 if c['gamma'] != 0. else 0)
        total += ffts * 5. * n * n * math.log2(n)
    per_rank = total / world
    mhz = (clocks or {}).get('sm_mhz') or 1965.
    nominal = 148 * 128 * 2 * mhz * 1e6 / 1e12
    achieved = per_rank / (ms_step / 1e3) / 1e12
    return {'algorithmic_per_step': total, 'achieved_tflops': achieved, 'fp32_nominal_tflops': nominal,
            'frac_of_nominal': achieved / nominal, 'counted': '5 N log2 N per transform; 10 transforms per '
            'point per damped step in the complex formulation (the real-storage packing does the step with 5, '
            'so this is an equivalent rate)'}


# DRAM bytes of one Dirac2D step of one replica at 512^2 (row + column pass, read + write), from
# the ncu capture summarised in profiles/dirac_passes_512.md (the replica fits in L2: one read of
# it per pass, the writes still in L2 when each kernel ends)
NCU_TRAFFIC_DIRAC = 16.917e6 + 0.002e6 + 16.822e6 + 0.0003e6


def make_dirac_instance(time_steps):
    from pywignercuda_b200 import GPU_Dirac2D

    class Coulomb(GPU_Dirac2D):
        def __init__(self):
            self.mass, self.c, self.hBar = 1., 137.036, 1.
            self.Potential_0_String = '-1./sqrt(x*x+y*y+0.5)'
            self.Potential_1_String = self.Potential_2_String = self.Potential_3_String = '0.'
            self.fileName = ''
            GPU_Dirac2D.__init__(self, (512, 512), (12., 12.), 1e-4, time_steps, 10 ** 9)
    return Coulomb()


def run_dirac(args, world, rank, local):
    """Dirac2D 512x512, c = 137.036, softened Coulomb, packet p0 = (5, 0), dt = 1e-4,
    complex128, R replicas in lock-step (dirac_run_many)."""
    import ctypes
    import torch
    from pywignercuda_b200 import _lib
    lib = _lib.load()
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    R = args.replicas
    insts = [make_dirac_instance(args.steps) for _ in range(R)]
    P0 = insts[0].Spinor_Particle_SpinUp((5., 0.), lambda x, y: np.exp(-(x * x + y * y) / 2.))
    Ps = [torch.from_numpy(np.ascontiguousarray(P0, dtype=np.complex128)).to(dev) for _ in range(R)]
    stream = torch.cuda.current_stream(dev)
    hs = (ctypes.c_void_p * R)(*[i._handle.value for i in insts])
    ps = (ctypes.c_void_p * R)(*[p.data_ptr() for p in Ps])
    _lib.check(lib.dirac_run_many(hs, ps, R, 0, args.warmup, None, stream.cuda_stream), 'warm-up')
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        _lib.check(lib.dirac_run_many(hs, ps, R, args.warmup, args.steps, None, stream.cuda_stream), 'timed')
        e1.record(stream)
        torch.cuda.synchronize()
    ms = barrier_max(world, e0.elapsed_time(e1))
    value = world * R * 512 * 512 * args.steps / (ms / 1e3)
    peak, peak_kind = peaks()
    achieved = 2 * 512 * 512 * 128 / (ms / 1e3 / (R * args.steps)) / 1e9   # 2 passes x 128 B per point
    # end to end: each replica's pinned host spinor in, host spinor and observables out, through
    # dirac_run_host (one untimed 1-step call first allocates each handle's device staging buffer)
    P0c = np.ascontiguousarray(P0, dtype=np.complex128)
    host_in = torch.from_numpy(P0c).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    obs_e2e = np.empty((args.steps, _lib.DIRAC_NOBS))
    for i in insts:
        _lib.check(lib.dirac_run_host(i._handle, host_in.data_ptr(), host_out.data_ptr(), 0, 1, None,
                                      stream.cuda_stream), 'e2e warm-up')
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for i in insts:
        _lib.check(lib.dirac_run_host(i._handle, host_in.data_ptr(), host_out.data_ptr(), 0, args.steps,
                                      _lib.dptr(obs_e2e), stream.cuda_stream), 'e2e')
    e2e_s = barrier_max(world, time.perf_counter() - t0)
    line = {'metric': 'Dirac2D spinor-pt-steps/s', 'value': value, 'unit': 'spinor-pt-steps/s',
            'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'c128',
            'data': 'synthetic',
            'config': {'workload': 'Dirac2D 512x512 c=137.036 softened Coulomb, p0=(5,0), dt=1e-4',
                       'replicas_per_gpu': R,
                       'l2': 'per-step working set %d MB > 126 MB L2' % (R * 16)},
            'e2e': {'value': world * R * 512 * 512 * args.steps / e2e_s, 'unit': 'spinor-pt-steps/s',
                    'h2d_bytes_per_step': R * P0c.nbytes / args.steps,
                    'd2h_bytes_per_step': R * (P0c.nbytes + obs_e2e.nbytes) / args.steps,
                    'note': 'one dirac_run_host call per replica, one after the other, pinned host spinors'},
            'roofline': {'bound': 'hbm', 'kernel': 'dirac_rowpass+dirac_colpass (step average)',
                         'algorithmic_bytes_per_point': 256, 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                         'frac': achieved / peak, 'peak_kind': peak_kind, 'traffic': NCU_TRAFFIC_DIRAC,
                         'traffic_per': 'step (row + column pass) of one replica, ncu at 512^2'},
            'gpu_launches': R * (2 * args.steps + 3), 'clocks': clk.summary()}
    if rank == 0 and args.cpu_baseline:
        from oracle.dirac2d import DiracOracle, DiracParams
        prm = DiracParams(512, 512, 12., 12., 1e-4, c=137.036, A0='-1./sqrt(x*x+y*y+0.5)')
        orc = DiracOracle(prm)
        t0, k = time.perf_counter(), 0
        while time.perf_counter() - t0 < 10. or k < 1:
            orc.run(P0c, 1)
            k += 1
        dt_cpu = time.perf_counter() - t0
        line['cpu_baseline'] = {'value': 512 * 512 * k / dt_cpu, 'unit': 'spinor-pt-steps/s',
                                'cores': os.cpu_count(), 'kind': 'port',
                                'sample': '%d steps of the oracle (numpy + scipy.fft) at 512^2, same instance' % k}
    if rank == 0:
        print(json.dumps(line))


D3N = 256
D3_BYTES = 512   # per grid point per step: 4 passes x (read + write of 4 complex128 components)
# DRAM bytes of one step at 256^3 from one ncu capture (dram__bytes rate x duration of each of the
# four passes, profiles/dirac3d_passes_256cube.md)
NCU_TRAFFIC_D3 = 2.090e9 + 2.088e9 + 2.096e9 + 2.089e9


def make_dirac3d_instance(n, time_steps):
    from pywignercuda_b200 import GPU_Dirac3D

    class Coulomb3D(GPU_Dirac3D):
        def __init__(self):
            self.mass, self.c, self.hBar = 1., 137.036, 1.
            self.Potential_0_String = '-1./sqrt(x*x+y*y+z*z+0.5)'
            self.Potential_1_String = self.Potential_2_String = self.Potential_3_String = '0.'
            self.fileName = ''
            self.Compute_Ehrenfest_P = True
            GPU_Dirac3D.__init__(self, (n, n, n), (12., 12., 12.), 1e-4, time_steps, 10 ** 9)
    return Coulomb3D()


def run_dirac3d(args, world, rank, local):
    """Dirac3D 256^3 (a 1 GB spinor), c = 137.036, softened Coulomb, packet
    p0 = (5, 0, 1), dt = 1e-4, complex128, one instance per GPU (dirac3_run)."""
    import torch
    from pywignercuda_b200 import _lib
    from oracle.dirac3d import Dirac3DOracle, Dirac3DParams
    lib = _lib.load()
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    steps = args.steps
    inst = make_dirac3d_instance(D3N, steps)
    gauss = lambda x, y, z: np.exp(-(x * x + y * y + z * z) / 2.)
    P0 = np.ascontiguousarray(inst.Spinor_Particle_SpinUp((5., 0., 1.), gauss), dtype=np.complex128)
    psi = torch.from_numpy(P0).to(dev)
    stream = torch.cuda.current_stream(dev)
    obs = np.empty((max(steps, args.warmup), _lib.DIRAC3_NOBS))
    _lib.check(lib.dirac3_run(inst._handle, psi.data_ptr(), 0, args.warmup, 0, _lib.dptr(obs),
                              stream.cuda_stream), 'warm-up')
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        _lib.check(lib.dirac3_run(inst._handle, psi.data_ptr(), args.warmup, steps, _lib.WIG_RUN_CONTINUE, None,
                                  stream.cuda_stream), 'timed')
        e1.record(stream)
        torch.cuda.synchronize()
    ms = barrier_max(world, e0.elapsed_time(e1))
    npts = D3N ** 3
    value = world * npts * steps / (ms / 1e3)
    peak, peak_kind = peaks()
    achieved = D3_BYTES * npts / (ms / 1e3 / steps) / 1e9
    # end to end: pinned host spinor in, host spinor and observables out, through dirac3_run_host
    # (one untimed 1-step call first allocates the handle's device staging buffer)
    host_in = torch.from_numpy(P0).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    obs_e2e = np.empty((steps, _lib.DIRAC3_NOBS))
    _lib.check(lib.dirac3_run_host(inst._handle, host_in.data_ptr(), host_out.data_ptr(), 0, 1, 0, None,
                                   stream.cuda_stream), 'e2e warm-up')
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    _lib.check(lib.dirac3_run_host(inst._handle, host_in.data_ptr(), host_out.data_ptr(), 0, steps, 0,
                                   _lib.dptr(obs_e2e), stream.cuda_stream), 'e2e')
    e2e_s = barrier_max(world, time.perf_counter() - t0)
    line = {'metric': 'Dirac3D spinor-pt-steps/s', 'value': value, 'unit': 'spinor-pt-steps/s',
            'n_gpus': world, 'steps': steps, 'warmup': args.warmup, 'ms_per_step': ms / steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'c128',
            'data': 'synthetic',
            'config': {'workload': 'Dirac3D 256^3, [-12,12)^3, c=137.036 softened Coulomb, p0=(5,0,1), dt=1e-4',
                       'l2': 'spinor 1074 MB > 126 MB L2'},
            'e2e': {'value': world * npts * steps / e2e_s, 'unit': 'spinor-pt-steps/s',
                    'h2d_bytes_per_step': P0.nbytes / steps, 'd2h_bytes_per_step': (P0.nbytes + obs_e2e.nbytes) / steps},
            'roofline': {'bound': 'hbm', 'kernel': 'd3_xpass + 2 d3_ypass + d3_zpass (step average)',
                         'algorithmic_bytes_per_point': D3_BYTES, 'achieved': achieved, 'peak': peak,
                         'unit': 'GB/s', 'frac': achieved / peak, 'peak_kind': peak_kind,
                         'traffic': NCU_TRAFFIC_D3, 'traffic_per': 'step (4 launches), ncu at 256^3',
                         'algorithmic_bytes_per_step': D3_BYTES * npts},
            'gpu_launches': 4 * steps + 1, 'clocks': clk.summary()}
    if rank == 0 and args.cpu_baseline:
        n = 128
        prm = Dirac3DParams(n, n, n, 12., 12., 12., 1e-4, c=137.036, A0='-1./sqrt(x*x+y*y+z*z+0.5)')
        orc = Dirac3DOracle(prm)
        from oracle.dirac3d import spinor_particle_spin_up_3d
        P = spinor_particle_spin_up_3d(prm, (5., 0., 1.), gauss)
        t0, k = time.perf_counter(), 0
        while time.perf_counter() - t0 < 10. or k < 1:
            orc.run(P, 1, t_index0=k, normalise=(k == 0))
            k += 1
        dt_cpu = time.perf_counter() - t0
        line['cpu_baseline'] = {'value': n ** 3 * k / dt_cpu, 'unit': 'spinor-pt-steps/s',
                                'cores': os.cpu_count(), 'kind': 'port',
                                'sample': '%d steps of the oracle (numpy + scipy.fft) at 128^3, same physics' % k}
    if rank == 0:
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=1000)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--replicas', type=int, default=REPLICAS)
    ap.add_argument('--no-cpu-baseline', dest='cpu_baseline', action='store_false')
    ap.add_argument('--workload', default='batch', choices=['batch', 'c128', 'dirac', 'dirac3d', 'gp', 'shardcost',
                                                                'adjoint'])
    ap.add_argument('--profile-only', action='store_true',
                    help='batch workload: only the timed section (for profiler launch lists)')
    ap.add_argument('--precision', default='both', choices=['both', 'mixed', 'f32'],
                    help='batch workload: the precisions timed (profiling runs)')
    ap.add_argument('--warps', type=int, default=0, choices=[0, 2, 4, 8],
                    help='batch workload: fixed tile shape (warps per CTA) instead of autotuning (profiling runs)')
    ap.add_argument('--instances', type=int, default=0,
                    help='batch workload: instances per rank (default 64; profiling runs)')
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == 'reference':
        # host-only work on rank 0; the other ranks exit 0 without joining a process group
        run_reference(args, int(os.environ.get('WORLD_SIZE', '1')), int(os.environ.get('RANK', '0')))
        return
    world, rank, local = dist_setup()
    try:
        if args.workload == 'dirac':
            run_dirac(args, world, rank, local)
        elif args.workload == 'c128':
            run_c128(args, world, rank, local)
        elif args.workload == 'gp':
            run_gp(args, world, rank, local)
        elif args.workload == 'dirac3d':
            run_dirac3d(args, world, rank, local)
        elif args.workload == 'shardcost':
            run_shardcost(args, world, rank, local)
        elif args.workload == 'adjoint':
            run_adjoint(args, world, rank, local)
        else:
            run_batch(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == '__main__':
    main()
