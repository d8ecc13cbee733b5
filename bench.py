"""Benchmark: Wigner2D grid-point-steps per second on B200.

Workload: the 1024x1024 double-well Caldeira-Leggett instance (x, p in
[-12, 12), V = 0.05x^4 - x^2, gamma = 0.1, kT = 0.5 -> D_theta = 0.1,
f(p) = |p|, cat state at x = +-3, sigma 0.7, dt = 0.005), complex128, built
through the public drop-in class.  R = 16 independent replicas are stepped in
lock-step (wig_run_many): the per-step working set is 16 x 16 MB = 256 MB,
larger than the 126 MB L2, so no replica's state stays cached between its
steps.  One bench "step" = one propagation of every replica.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (launched by torchrun): every rank runs its own R replicas (weak
scaling, no data-path collective: the instances are independent); the
elapsed time is the max over ranks.  --impl reference times the oracle's
restatement of the reference's propagator (numpy + scipy.fft on all host
cores) on the same workload; rank 0 only.
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
# dram__bytes_read.sum + dram__bytes_write.sum per p-pass launch, from the ncu capture
# summarised in profiles/wig_ppass_c128_1024.md (None until a capture exists)
NCU_TRAFFIC_PPASS = None


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
                                          '--format=csv,noheader,nounits', '-lms', '200'],
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
    t = torch.tensor([value], dtype=torch.float64, device='cuda')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


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


def run_reference(args, world, rank):
    if rank != 0:
        return
    budget = 150.0
    # warm-up steps (untimed) then K timed steps, each one propagation of one instance
    rate, n, el, cores = cpu_baseline_run(max_seconds=min(budget, 1e9), min_steps=args.steps,
                                          max_steps=args.steps)
    line = {'metric': METRIC, 'value': rate, 'unit': UNIT, 'n_gpus': args.gpus, 'steps': n,
            'warmup': args.warmup, 'ms_per_step': 1e3 * el / n, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'c128', 'data': 'synthetic',
            'impl': 'reference',
            'config': {'workload': 'Wigner2D 1024x1024 double well, Caldeira-Leggett, complex128',
                       'form': 'CPU restatement of GPU_Wigner2D_FFT.Run (numpy + scipy.fft)'},
            'cpu_baseline': {'value': rate, 'unit': UNIT, 'cores': cores, 'kind': 'port',
                             'sample': '%d propagations of one 1024x1024 instance' % n},
            'e2e': {'value': rate, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line))


def run_ours(args, world, rank, local):
    import ctypes
    import torch
    from pywignercuda_b200 import _lib
    lib = _lib.load()
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    R = args.replicas
    insts = [make_instance(args.steps) for _ in range(R)]
    W0 = cat_state(insts[0])
    Ws = [torch.from_numpy(W0.astype(np.complex128)).to(dev) for _ in range(R)]
    stream = torch.cuda.current_stream(dev)
    hs = (ctypes.c_void_p * R)(*[i._handle.value for i in insts])
    ws = (ctypes.c_void_p * R)(*[w.data_ptr() for w in Ws])
    obs = [np.empty((args.steps + 1, _lib.WIG_NOBS)) for _ in range(R)]
    obs_p = (_lib._DP * R)(*[_lib.dptr(o) for o in obs])
    warm = [np.empty((args.warmup + 1, _lib.WIG_NOBS)) for _ in range(R)]
    warm_p = (_lib._DP * R)(*[_lib.dptr(o) for o in warm])
    _lib.check(lib.wig_run_many(hs, ws, R, 0, args.warmup, 0, warm_p, stream.cuda_stream), 'warm-up')
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flags = _lib.WIG_RUN_CONTINUE | _lib.WIG_RUN_PROFILE
    with ClockSampler(local) as clk:
        e0.record(stream)
        _lib.check(lib.wig_run_many(hs, ws, R, args.warmup, args.steps, flags, obs_p, stream.cuda_stream),
                   'timed run')
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = barrier_max(world, e0.elapsed_time(e1))
    pts_steps = world * R * NX * NP * args.steps
    value = pts_steps / (ms / 1e3)
    # per-kernel device time (CUDA events around every launch, same stream)
    x_ms = p_ms = 0.
    launches = 0
    for i in insts:
        out = (ctypes.c_double * 2)()
        cnt = ctypes.c_int64()
        _lib.check(lib.wig_profile(i._handle, out, ctypes.byref(cnt)), 'wig_profile')
        x_ms += out[0]
        p_ms += out[1]
        launches += cnt.value
    dom, dom_ms = ('wig_ppass', p_ms) if p_ms >= x_ms else ('wig_xpass', x_ms)
    avg_s = dom_ms / launches / 1e3
    peak, peak_kind = peaks()
    achieved = PASS_BYTES / avg_s / 1e9
    # physics check of the timed run: the norm stays 1, no NaN
    norm_err = max(float(np.max(np.abs(o[:, 0] - 1.))) for o in obs)
    # ---------------- e2e: host buffers in, host buffers out, through the C ABI
    hin = [torch.from_numpy(W0.astype(np.complex128)).pin_memory() for _ in range(R)]
    hout = [torch.empty_like(h).pin_memory() for h in hin]
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for w, h in zip(Ws, hin):
        w.copy_(h, non_blocking=True)
    _lib.check(lib.wig_run_many(hs, ws, R, 0, args.steps, 0, obs_p, stream.cuda_stream), 'e2e run')
    for w, h in zip(Ws, hout):
        h.copy_(w, non_blocking=True)
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = barrier_max(world, max(f0.elapsed_time(f1), 1e3 * (time.perf_counter() - t0)))
    grid_bytes = NX * NP * 16
    line = {
        'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': ms / args.steps, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'c128', 'data': 'synthetic',
        'config': {'workload': 'Wigner2D 1024x1024 double well V=0.05x^4-x^2, Caldeira-Leggett gamma=0.1 '
                               'D_theta=0.1 f=|p|, cat state, dt=0.005',
                   'form': 'plain complex128 (the FP32 batched form is not built yet)',
                   'replicas_per_gpu': R, 'parallelism': 'independent instances, one process per GPU',
                   'l2': 'per-step working set %d MB > 126 MB L2' % (R * grid_bytes >> 20),
                   'max_abs_norm_error': norm_err},
        'roofline': {'bound': 'hbm', 'kernel': dom, 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                     'frac': achieved / peak, 'peak_kind': peak_kind,
                     'algorithmic_bytes_per_launch': PASS_BYTES, 'avg_launch_us': avg_s * 1e6,
                     'x_pass_us': x_ms / launches * 1e3, 'p_pass_us': p_ms / launches * 1e3,
                     'traffic': NCU_TRAFFIC_PPASS},
        'e2e': {'value': world * R * NX * NP * args.steps / (e2e_ms / 1e3), 'unit': UNIT,
                'h2d_bytes_per_step': R * grid_bytes / args.steps,
                'd2h_bytes_per_step': (R * grid_bytes + R * (args.steps + 1) * 11 * 8) / args.steps,
                'note': 'one Run()-style call per bench: upload W_init, K propagations, download W_end '
                        'and the observables; bytes are per propagation step'},
        'gpu_launches': R * (2 * args.steps + 3),
        'clocks': clk.summary(),
    }
    if rank == 0 and args.cpu_baseline:
        rate, n, el, cores = cpu_baseline_run(max_seconds=15.0)
        line['cpu_baseline'] = {'value': rate, 'unit': UNIT, 'cores': cores, 'kind': 'port',
                                'sample': '%d propagations of one 1024x1024 instance (%.1f s)' % (n, el)}
    if rank == 0:
        print(json.dumps(line))
    del insts


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
    line = {'metric': 'Dirac2D spinor-pt-steps/s', 'value': value, 'unit': 'spinor-pt-steps/s',
            'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'c128',
            'data': 'synthetic',
            'config': {'workload': 'Dirac2D 512x512 c=137.036 softened Coulomb, p0=(5,0), dt=1e-4',
                       'replicas_per_gpu': R,
                       'l2': 'per-step working set %d MB > 126 MB L2' % (R * 16)},
            'roofline': {'bound': 'hbm', 'kernel': 'dirac_rowpass+dirac_colpass (step average)',
                         'achieved': achieved, 'peak': peak, 'unit': 'GB/s', 'frac': achieved / peak,
                         'peak_kind': peak_kind, 'traffic': None},
            'gpu_launches': R * (2 * args.steps + 3), 'clocks': clk.summary()}
    if rank == 0:
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=200)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--replicas', type=int, default=REPLICAS)
    ap.add_argument('--no-cpu-baseline', dest='cpu_baseline', action='store_false')
    ap.add_argument('--workload', default='wigner', choices=['wigner', 'dirac'])
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup()
    try:
        if args.impl == 'reference':
            run_reference(args, world, rank)
        elif args.workload == 'dirac':
            run_dirac(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == '__main__':
    main()
