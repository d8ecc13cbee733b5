"""Build the native library ``libwigner_b200.so`` (nvcc, sm_100a).

Steps:
1. inline the device headers of each JIT entry file (``csrc/wig_jit_*.cuh``)
   into ``csrc/wig_device_src.inc`` as C++ raw string literals -- the source
   NVRTC compiles per propagator instance;
2. ``nvcc -gencode arch=compute_100a,code=sm_100a -shared`` of ``csrc/*.cu``
   into ``pywignercuda_b200/libwigner_b200.so`` (CUDA runtime linked
   statically; NVRTC and the driver are reached at run time, so the library
   loads on machines without a GPU).

Usage: ``python -m pywignercuda_b200.build`` (or ``build()`` from Python).
"""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'libwigner_b200.so')
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')

# generated include -> {string name: JIT entry file}
JIT_SOURCES = {'wig_device_src.inc': {'kJitWignerSource': 'wig_jit_wigner.cuh', 'kJitDiracSource': 'wig_jit_dirac.cuh',
                                      'kJitBatchSource': 'wig_jit_batch.cuh'},
               'wig_adjoint_src.inc': {'kJitAdjointSource': 'wig_jit_adjoint.cuh'},
               'wig_dirac3_src.inc': {'kJitDirac3Source': 'wig_jit_dirac3.cuh'}}


def inline(fn, seen=None):
    seen = set() if seen is None else seen
    out = []
    with open(os.path.join(CSRC, fn)) as f:
        for line in f:
            m = re.match(r'\s*#include "(.*)"', line)
            if m:
                if m.group(1) not in seen:
                    seen.add(m.group(1))
                    out.append(inline(m.group(1), seen))
                continue
            if line.strip() == '#pragma once':
                continue
            out.append(line)
    return ''.join(out)


def write_inc():
    for inc, srcs in JIT_SOURCES.items():
        parts = ['// generated by pywignercuda_b200/build.py -- do not edit\n']
        for name, fn in srcs.items():
            src = inline(fn)
            assert ')WIGSRC"' not in src
            # split into chunks below the 64 KiB string-literal limit of some compilers
            chunks = [src[i:i + 30000] for i in range(0, len(src), 30000)]
            body = '\n'.join('R"WIGSRC(%s)WIGSRC"' % c for c in chunks)
            parts.append('static const char %s[] =\n%s;\n' % (name, body))
        path = os.path.join(CSRC, inc)
        text = ''.join(parts)
        if not os.path.exists(path) or open(path).read() != text:
            with open(path, 'w') as f:
                f.write(text)


def build(verbose=False):
    write_inc()
    sources = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith('.cu')]
    deps = sources + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(('.cuh', '.inc', '.h'))]
    deps.append(os.path.join(os.path.dirname(HERE), 'include', 'wigner_b200.h'))
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    cmd = [NVCC, '-O3', '-std=c++17', '-shared', '-Xcompiler', '-fPIC', '-lineinfo',
           '-gencode', 'arch=compute_100a,code=sm_100a', '-Xptxas', '-v',
           '-o', LIB + '.tmp'] + sources + ['-ldl']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('nvcc failed:\n' + r.stdout + r.stderr)
    if verbose:
        print(r.stdout + r.stderr)
    os.replace(LIB + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    print(build(verbose='-v' in sys.argv))
