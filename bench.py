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
                  [--workload batch|c128|dirac|dirac3d|gp]

N > 1 (torchrun): the batch has 64 N instances partitioned by cost across the
ranks (weak scaling; no data-path collective, the observables are gathered to
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
# L2: the capture shows one read of it) and profiles/wigb_passes_batch64.md (the 64-instance
# batch, 187 MB of state)
NCU_TRAFFIC_PPASS = 16.94e6 + 0.04e6
NCU_TRAFFIC_BATCH = 188.0e6 + 129.2e6


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
    flags = _lib.WIG_RUN_CONTINUE | _lib.WIG_RUN_PROFILE
    with ClockSampler(local) as clk:
        e0.record(stream)
        _lib.check(lib.wig_run_many(hs, ws, R, args.warmup, steps, flags, obs_p, stream.cuda_stream), 'timed')
        e1.record(stream)
        torch.cuda.synchronize()
    ms = barrier_max(world, e0.elapsed_time(e1))
    value = world * R * NX * NP * steps / (ms / 1e3)
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


def run_batch(args, world, rank, local):
    """Headline: the FP32 batched form on the 64-instance mixed-grid batch.  With
    N ranks the batch has 64 N instances (the same generator; N = 1 is the
    configuration itself) partitioned by cost across the ranks (weak scaling);
    each rank runs its share, the observables are gathered to rank 0."""
    import torch
    from pywignercuda_b200.batch import WignerBatch, instance
    from pywignercuda_b200.shard import gather_observables, partition
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    cases_all = batch_config(count=64 * world)
    parts = partition([dict(n_x=c['n'], n_p=c['n'], gamma=c['gamma']) for c in cases_all], world)
    cases = [cases_all[i] for i in parts[rank]]
    grand_total = sum(c['n'] * c['n'] for c in cases_all)
    batch = WignerBatch([instance(c['n'], x_amplitude=10., dt=DT, gamma=c['gamma'], d_theta=c['d_theta'],
                                  v4=c['a'], v2=c['b']) for c in cases])
    states = [coherent_state(c['n'], c['x0'], c['p0']) for c in cases]
    total = batch.total
    stream = torch.cuda.current_stream(dev)
    scratch = batch.pack(states)
    warps, tune_ms = batch.autotune(scratch, probe_steps=3)
    del scratch
    K = args.steps
    W = batch.pack(states)
    batch.run(W, args.warmup)                                           # normalises
    batch.run(W, K, continue_run=True, observables=False)               # captures the K-step graph
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        batch.run(W, K, continue_run=True)                              # graph replay; obs D2H included
        e1.record(stream)
        torch.cuda.synchronize()
    ms = barrier_max(world, e0.elapsed_time(e1))
    value = grand_total * K / (ms / 1e3)
    if args.profile_only:
        if rank == 0:
            print(json.dumps({'metric': METRIC, 'value': value, 'unit': UNIT, 'steps': K, 'warps': warps,
                              'note': 'profile-only run (timed section only)'}))
        return
    # per-pass device time (a short non-graph run with events around every launch)
    nprof = min(K, 20)
    batch.run(W, nprof, continue_run=True, graph=False, observables=False, profile=True)
    x_ms, p_ms, nl = batch.profile()
    peak, peak_kind = peaks()
    pass_bytes = total * 8 * 2                                        # complex64 read + write per pass
    dom, dom_ms = ('wigb_ppass', p_ms) if p_ms >= x_ms else ('wigb_xpass', x_ms)
    achieved = pass_bytes / (dom_ms / nl / 1e3) / 1e9
    # FP32 drift against complex128 on every instance (fresh run, same steps)
    nval = min(K, 200)
    Wv = batch.pack(states)
    obs32 = batch.run(Wv, nval, graph=False)
    obs64 = c128_reference_obs(cases, nval, dev)
    norm_err = float(np.max(np.abs(obs32[:, :, 0] - obs64[:, :, 0])))
    energy_abs = np.max(np.abs(obs32[:, :, 9] - obs64[:, :, 9]), axis=1)
    # scale of H(x, p) over each instance's grid: the FP32 FFT noise is weighted by it
    hrange = np.array([10. ** 2 / 2. + abs(c['a']) * 10. ** 4 + abs(c['b']) * 10. ** 2 for c in cases])
    energy_err = float(np.max(energy_abs))
    energy_err_h = float(np.max(energy_abs / hrange))
    del Wv
    # e2e: pinned host state in, run, host state and observables out, all timed
    hin = torch.from_numpy(np.concatenate([s.astype(np.complex64).ravel() for s in states])).pin_memory()
    hout = torch.empty_like(hin).pin_memory()
    Wd = torch.empty(total, dtype=torch.complex64, device=dev)
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
    c128 = run_c128(args, world, rank, local, steps=min(K, 100), emit=False)
    line = {
        'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': K, 'warmup': args.warmup,
        'ms_per_step': ms / K, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f32 (FP64 phase arguments and observables)', 'data': 'synthetic',
        'config': {'workload': '64 Wigner2D instances, square grids from {128,256,512,1024} (default_rng(0)), '
                               'V=a x^4+b x^2, Caldeira-Leggett, coherent states, dt=0.005',
                   'form': 'FP32 batched, one x-pass + one p-pass launch per step, CUDA graph',
                   'instances': len(cases_all), 'instances_per_rank': [len(p) for p in parts],
                   'grid_points': grand_total, 'warps_per_cta': warps,
                   'autotune_ms': tune_ms,
                   'parallelism': 'instances partitioned by cost across ranks, one process per GPU, '
                                  'observables gathered to rank 0 (no data-path collective)',
                   'l2': 'state %d MB > 126 MB L2' % (total * 8 >> 20)},
        'plain_c128': c128,
        'ratio_fp32_batched_vs_c128': value / c128['value'],
        'drift_vs_fp64': {'steps': nval, 'norm_max_abs': norm_err, 'energy_max_abs': energy_err,
                          'energy_max_rel_to_H_range': energy_err_h,
                          'reference': 'complex128 drop-in path, exact constants, same instances'},
        'flops': batch_flops(cases_all, world, ms / K, clk.summary()),
        'roofline': {'bound': 'hbm', 'kernel': dom, 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                     'frac': achieved / peak, 'peak_kind': peak_kind, 'algorithmic_bytes_per_launch': pass_bytes,
                     'avg_launch_us': dom_ms / nl * 1e3, 'x_pass_us': x_ms / nl * 1e3, 'p_pass_us': p_ms / nl * 1e3,
                     'traffic': NCU_TRAFFIC_BATCH},
        'e2e': {'value': grand_total * K / (e2e_ms / 1e3), 'unit': UNIT,
                'h2d_bytes_per_step': grand_total * 8 / K,
                'd2h_bytes_per_step': (grand_total * 8 + len(cases_all) * (K + 1) * 11 * 8) / K,
                'note': 'one run call: upload the packed states, K propagations, download states and '
                        'observables; bytes per propagation step'},
        'gpu_launches': 2 * K + 2,
        'clocks': clk.summary(),
    }
    if rank == 0 and args.cpu_baseline:
        rate, n, el, cores, what = cpu_batch_sample(cases, max_seconds=15.0)
        line['cpu_baseline'] = {'value': rate, 'unit': UNIT, 'cores': cores, 'kind': 'port',
                                'sample': what + ' (%.1f s)' % el}
    if rank == 0:
        print(json.dumps(line))


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
    ap.add_argument('--workload', default='batch', choices=['batch', 'c128', 'dirac', 'dirac3d', 'gp'])
    ap.add_argument('--profile-only', action='store_true',
                    help='batch workload: only the timed section (for profiler launch lists)')
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
        else:
            run_batch(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == '__main__':
    main()
