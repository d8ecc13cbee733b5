"""bench.py's reference arm on the host: the JSON line it prints and its
behaviour on ranks other than 0.  The GPU arm is exercised by the GPU tests
and the bench itself."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(extra_env=None, timeout=300):
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference',
                           '--steps', '1', '--warmup', '3'],
                          capture_output=True, text=True, timeout=timeout, env=env, cwd=ROOT)


def test_reference_arm_line():
    p = _run()
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith('{')]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ('metric', 'value', 'unit', 'n_gpus', 'steps', 'warmup', 'ms_per_step', 'higher_is_better',
              'scaling', 'vs_baseline', 'dtype', 'data', 'config', 'cpu_baseline', 'e2e'):
        assert k in d, k
    assert d['impl'] == 'reference'
    assert d['metric'] == 'Wigner2D grid-pt-steps/s: FP32 batched vs plain complex128 at stated error'
    assert d['unit'] == 'grid-pt-steps/s' and d['higher_is_better'] is True
    assert d['value'] > 0 and d['steps'] >= 2 and d['warmup'] >= 3
    assert d['cpu_baseline']['kind'] == 'port' and d['cpu_baseline']['cores'] >= 1
    assert d['cpu_baseline']['value'] == d['value']
    assert d['e2e'] == {'value': d['value'], 'unit': d['unit'], 'h2d_bytes_per_step': 0,
                        'd2h_bytes_per_step': 0}


def test_reference_arm_other_ranks_exit_quietly():
    p = _run({'WORLD_SIZE': '2', 'RANK': '1', 'LOCAL_RANK': '1'}, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert not [ln for ln in p.stdout.splitlines() if ln.startswith('{')]


def test_notebook_cpu_baseline_sample():
    """The second CPU baseline: the notebook's own real-FFT Strang propagator at its
    512^2 configuration (a short sample here)."""
    import bench
    r = bench.cpu_notebook_sample(steps=2, repeats=1, warmup=1)
    assert r['value'] > 0 and r['unit'] == bench.UNIT and r['kind'] == 'port' and r['cores'] >= 1


def _undefined_names(path):
    import ast
    import builtins
    tree = ast.parse(open(path).read())
    defined = {n.id for n in ast.walk(tree) if isinstance(n, ast.Name) and isinstance(n.ctx, ast.Store)}
    defined |= {n.name for n in ast.walk(tree) if isinstance(n, (ast.FunctionDef, ast.ClassDef))}
    defined |= {n.arg for n in ast.walk(tree) if isinstance(n, ast.arg)}
    for n in ast.walk(tree):
        if isinstance(n, (ast.Import, ast.ImportFrom)):
            defined |= {(a.asname or a.name).split('.')[0] for a in n.names}
        if isinstance(n, ast.ExceptHandler) and n.name:
            defined.add(n.name)
    used = {n.id for n in ast.walk(tree) if isinstance(n, ast.Name) and isinstance(n.ctx, ast.Load)}
    return sorted(u for u in used - defined if not hasattr(builtins, u) and u != '__file__')


def test_bench_and_package_names_are_defined():
    """Every name bench.py and the package's modules read is defined, imported, a
    parameter or a builtin: their GPU paths only run on a GPU, so a missing
    module-level name would otherwise surface there first."""
    paths = [os.path.join(ROOT, 'bench.py')]
    pkg = os.path.join(ROOT, 'pywignercuda_b200')
    paths += [os.path.join(pkg, f) for f in sorted(os.listdir(pkg)) if f.endswith('.py')]
    for p in paths:
        assert not _undefined_names(p), (p, _undefined_names(p))
