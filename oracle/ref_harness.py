"""Run the reference's own host code on the CPU (TEST INFRASTRUCTURE ONLY).

The reference (cabrer7/PyWignerCUDA) is Python 2 + PyCUDA and cannot be
imported under Python 3 as it stands.  This harness:

1. reads a reference module's source text from the reference checkout named by
   the environment variable ``PYWIGNER_REFERENCE`` (required), expands its tabs
   the way the Python 2 tokenizer does (stops every 8 columns), turns ``print``
   statements into calls and ``np.float(`` into ``float(`` -- nothing else is
   changed -- and executes it as a module;
2. installs fake ``pycuda`` / ``cufft_wrapper`` / ``h5py`` / ``matplotlib``
   modules for that execution:

   * ``pycuda.compiler.SourceModule`` takes the reference's CUDA-C kernel
     strings *as the reference formats them* (``%f`` constants, user expression
     strings pasted in) and compiles them for the CPU with g++ against a tiny
     shim header (``pycuda::complex`` -> ``std::complex``, ``threadIdx`` /
     ``blockIdx`` as globals, a generated launcher that loops over the grid);
     the shared objects go to ``oracle/_ref/`` (git-ignored);
   * ``pycuda.gpuarray`` is a numpy-backed array with PyCUDA's operator
     semantics (``x /= s`` multiplies by ``1/s``, ``dot`` does not conjugate);
   * ``cufft_wrapper`` plans map to ``numpy.fft`` along the same axes, forward
     e^{-i} and unnormalised inverse, as cuFFT's Z2Z;
   * ``h5py.File`` keeps datasets in a dict so frames can be read back.

cuFFT itself is a closed library; its DFT is restated by ``numpy.fft`` (the
only stand-in in the chain).  Everything else that runs -- grids, constant
formatting, kernels, loop order, reductions, normalisations -- is the
reference's own code.  The harness is used only to generate the golden
fixtures in ``tests/golden`` (``tests/golden/make_golden.py``) and to validate
the restated oracle against them; it never runs on the GPU box.
"""
import ctypes
import hashlib
import io
import os
import re
import subprocess
import sys
import types
import contextlib

import numpy as np

REF_ROOT = os.environ.get('PYWIGNER_REFERENCE', '')
HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, '_ref')

# ----------------------------------------------------------------------------
# Python 2 -> 3 source conversion (print statements, tabs, np.float)
# ----------------------------------------------------------------------------
_PRINT_RE = re.compile(r'^(\s*)print\b(?!\s*\()(.*)$')


def py2_to_py3(src):
    out = []
    for line in src.splitlines():
        line = line.expandtabs(8)
        m = _PRINT_RE.match(line)
        if m:
            body = m.group(2).strip()
            line = '%sprint(%s)' % (m.group(1), body)
        line = re.sub(r'\bnp\.float\(', 'float(', line)
        out.append(line)
    return '\n'.join(out) + '\n'


# ----------------------------------------------------------------------------
# CPU compilation of the reference's CUDA-C kernel strings
# ----------------------------------------------------------------------------
SHIM = r'''
// CPU stand-ins for the CUDA / PyCUDA names the reference's kernels use.
#include <complex>
#include <cmath>
using namespace std;
namespace pycuda {
template <class T> using complex = std::complex<T>;
template <class T> inline T real(const std::complex<T>& z) { return z.real(); }
template <class T> inline T imag(const std::complex<T>& z) { return z.imag(); }
template <class T> inline std::complex<T> conj(const std::complex<T>& z) { return std::conj(z); }
}
struct harness_uint3 { unsigned x, y, z; };
static harness_uint3 threadIdx, blockIdx, blockDim, gridDim;
#define __global__
#define __device__ static inline
#define __constant__ static const
'''

_GLOBAL_RE = re.compile(r'__global__\s+void\s+(\w+)\s*\(([^)]*)\)', re.S)


def _params(plist):
    params = []
    for p in plist.split(','):
        p = ' '.join(p.split())
        if not p:
            continue
        m = re.match(r'(.*?)(\w+)$', p)
        typ, name = m.group(1).strip(), m.group(2)
        params.append((typ, name))
    return params


def _launcher(name, params):
    args = []
    for i, (typ, _) in enumerate(params):
        if '*' in typ:
            args.append('(%s)args[%d]' % (typ, i))
        else:
            args.append('*(%s*)args[%d]' % (typ, i))
    return r'''
extern "C" void harness_launch_%(n)s(unsigned gx, unsigned gy, unsigned gz,
                                     unsigned bx, unsigned by, unsigned bz, void** args) {
  gridDim.x = gx; gridDim.y = gy; gridDim.z = gz;
  blockDim.x = bx; blockDim.y = by; blockDim.z = bz;
  for (unsigned kz = 0; kz < gz; ++kz) for (unsigned ky = 0; ky < gy; ++ky)
  for (unsigned kx = 0; kx < gx; ++kx) {
    blockIdx.x = kx; blockIdx.y = ky; blockIdx.z = kz;
    for (unsigned tz = 0; tz < bz; ++tz) for (unsigned ty = 0; ty < by; ++ty)
    for (unsigned tx = 0; tx < bx; ++tx) {
      threadIdx.x = tx; threadIdx.y = ty; threadIdx.z = tz;
      %(n)s(%(a)s);
    }
  }
}
''' % dict(n=name, a=', '.join(args))


class _CpuKernel:
    def __init__(self, lib, name, params):
        self.fn = getattr(lib, 'harness_launch_' + name)
        self.fn.restype = None
        self.params = params

    def __call__(self, *args, block=(1, 1, 1), grid=(1, 1)):
        assert len(args) == len(self.params), (args, self.params)
        keep = []
        ptrs = (ctypes.c_void_p * len(args))()
        for i, (a, (typ, _)) in enumerate(zip(args, self.params)):
            if '*' in typ:
                assert isinstance(a, GPUArray)
                ptrs[i] = a.a.ctypes.data
            else:
                if 'double' in typ:
                    v = ctypes.c_double(float(a))
                elif 'int' in typ:
                    v = ctypes.c_int(int(a))
                else:
                    raise TypeError(typ)
                keep.append(v)
                ptrs[i] = ctypes.addressof(v)
        g = tuple(int(x) for x in grid) + (1,) * (3 - len(grid))
        b = tuple(int(x) for x in block) + (1,) * (3 - len(block))
        self.fn(ctypes.c_uint(g[0]), ctypes.c_uint(g[1]), ctypes.c_uint(g[2]),
                ctypes.c_uint(b[0]), ctypes.c_uint(b[1]), ctypes.c_uint(b[2]), ptrs)


class SourceModule:
    """CPU build of a reference kernel string (``pycuda.compiler.SourceModule``)."""

    def __init__(self, source, arch=None, **kw):
        src = source.replace('#include <pycuda-complex.hpp>', '')
        kernels = [(m.group(1), _params(m.group(2))) for m in _GLOBAL_RE.finditer(src)]
        full = SHIM + src + ''.join(_launcher(n, p) for n, p in kernels)
        h = hashlib.sha1(full.encode()).hexdigest()[:16]
        os.makedirs(BUILD_DIR, exist_ok=True)
        so = os.path.join(BUILD_DIR, 'refkern_%s.so' % h)
        if not os.path.exists(so):
            cpp = so[:-3] + '.cpp'
            with open(cpp, 'w') as f:
                f.write(full)
            subprocess.check_call(['g++', '-O2', '-std=c++17', '-shared', '-fPIC',
                                   '-ffp-contract=off', '-w', '-o', so + '.tmp', cpp])
            os.replace(so + '.tmp', so)
        lib = ctypes.CDLL(so)
        self.kernels = {n: _CpuKernel(lib, n, p) for n, p in kernels}

    def get_function(self, name):
        return self.kernels[name]


# ----------------------------------------------------------------------------
# numpy-backed gpuarray with PyCUDA operator semantics
# ----------------------------------------------------------------------------
class GPUArray:
    def __init__(self, a):
        self.a = a

    # -- PyCUDA attributes used by the reference
    dtype = property(lambda s: s.a.dtype)
    shape = property(lambda s: s.a.shape)
    size = property(lambda s: s.a.size)
    gpudata = property(lambda s: s.a.ctypes.data)
    ptr = property(lambda s: s.a.ctypes.data)
    mem_size = property(lambda s: s.a.size)

    def get(self):
        return self.a.copy()

    def copy(self):
        return GPUArray(np.array(self.a, copy=True))

    def conj(self):
        return GPUArray(np.conj(self.a))

    def __abs__(self):
        return GPUArray(np.abs(self.a))

    def __pow__(self, e):
        return GPUArray(np.power(self.a, e))

    @staticmethod
    def _v(o):
        return o.a if isinstance(o, GPUArray) else o

    def __mul__(self, o):
        return GPUArray(self.a * self._v(o))

    __rmul__ = __mul__

    def __add__(self, o):
        return GPUArray(self.a + self._v(o))

    __radd__ = __add__

    def __sub__(self, o):
        return GPUArray(self.a - self._v(o))

    def __neg__(self):
        return GPUArray(-self.a)

    def __truediv__(self, o):
        if isinstance(o, GPUArray):
            return GPUArray(self.a / o.a)
        return GPUArray(self.a * (1 / o))

    def __imul__(self, o):
        self.a *= self._v(o)
        return self

    def __iadd__(self, o):
        self.a += self._v(o)
        return self

    def __isub__(self, o):
        self.a -= self._v(o)
        return self

    def __itruediv__(self, o):
        # PyCUDA: x /= s  ->  x = (1/s) * x
        if isinstance(o, GPUArray):
            self.a /= o.a
        elif o != 1:
            self.a *= (1 / o)
        return self


def _gpuarray_module():
    m = types.ModuleType('pycuda.gpuarray')
    m.GPUArray = GPUArray
    m.to_gpu = lambda a: GPUArray(np.array(a, copy=True))
    m.empty_like = lambda g: GPUArray(np.empty_like(g.a))
    m.zeros_like = lambda g: GPUArray(np.zeros_like(g.a))
    m.empty = lambda shape, dtype=np.float64: GPUArray(np.empty(shape, dtype))
    m.zeros = lambda shape, dtype=np.float64: GPUArray(np.zeros(shape, dtype))
    m.sum = lambda g: GPUArray(np.array(np.sum(g.a)))
    m.dot = lambda a, b: GPUArray(np.array(np.sum(a.a * b.a)))
    return m


# ----------------------------------------------------------------------------
# cufft_wrapper stand-in
# ----------------------------------------------------------------------------
def _cufft_module():
    m = types.ModuleType('cufft_wrapper')

    class _Plan:
        def __init__(self, axes):
            self.axes = axes
            self.handle = 0

    def Plan_Z2Z(shape, batch=1):
        return _Plan(tuple(range(-len(shape), 0)))

    def Plan_Z2Z_2D_Axis0(shape):
        return _Plan((0,))

    def Plan_Z2Z_2D_Axis1(shape):
        return _Plan((1,))

    def fft_Z2Z(x, y, plan):
        y.a[...] = np.fft.fftn(x.a, axes=plan.axes)

    def ifft_Z2Z(x, y, plan):
        y.a[...] = np.fft.ifftn(x.a, axes=plan.axes, norm='forward')

    m.Plan_Z2Z, m.Plan_Z2Z_2D_Axis0, m.Plan_Z2Z_2D_Axis1 = Plan_Z2Z, Plan_Z2Z_2D_Axis0, Plan_Z2Z_2D_Axis1
    m.Plan_C2C = Plan_Z2Z
    m.fft_Z2Z, m.ifft_Z2Z = fft_Z2Z, ifft_Z2Z
    m.cufftDestroy = lambda h: None
    return m


# ----------------------------------------------------------------------------
# h5py / matplotlib stand-ins
# ----------------------------------------------------------------------------
H5_FILES = {}


class _H5File(dict):
    def __init__(self, name, mode=None, **kw):
        super().__init__()
        H5_FILES[name] = self

    def create_dataset(self, name, data=None, **kw):
        self[name] = np.array(data, copy=True)

    def __setitem__(self, k, v):
        super().__setitem__(k, np.array(v, copy=True) if not isinstance(v, str) else v)

    def close(self):
        pass


def _fake_modules():
    pycuda = types.ModuleType('pycuda')
    pycuda.__path__ = []
    gpuarray = _gpuarray_module()
    driver = types.ModuleType('pycuda.driver')
    driver.mem_get_info = lambda: (4 << 30, 5 << 30)
    driver.memcpy_dtod = lambda *a, **k: None
    autoinit = types.ModuleType('pycuda.autoinit')
    compiler = types.ModuleType('pycuda.compiler')
    compiler.SourceModule = SourceModule
    pycuda.gpuarray, pycuda.driver, pycuda.autoinit, pycuda.compiler = gpuarray, driver, autoinit, compiler
    h5py = types.ModuleType('h5py')
    h5py.File = _H5File
    mpl = types.ModuleType('matplotlib')
    mpl.__path__ = []
    plt = types.ModuleType('matplotlib.pyplot')
    colors = types.ModuleType('matplotlib.colors')
    mpl.pyplot, mpl.colors, mpl.rcParams = plt, colors, {}
    return {'pycuda': pycuda, 'pycuda.gpuarray': gpuarray, 'pycuda.driver': driver,
            'pycuda.autoinit': autoinit, 'pycuda.compiler': compiler,
            'cufft_wrapper': _cufft_module(), 'h5py': h5py, 'matplotlib': mpl,
            'matplotlib.pyplot': plt, 'matplotlib.colors': colors, 'pylab': plt}


_MODULE_CACHE = {}


def load_reference_module(name):
    """Execute ``<reference>/<name>.py`` (converted as described above) with the
    fake modules installed; returns the module object."""
    if name in _MODULE_CACHE:
        return _MODULE_CACHE[name]
    if not REF_ROOT or not os.path.isdir(REF_ROOT):
        raise RuntimeError('set PYWIGNER_REFERENCE to the reference checkout (cabrer7/PyWignerCUDA)')
    path = os.path.join(REF_ROOT, name + '.py')
    with open(path) as f:
        src = py2_to_py3(f.read())
    fakes = _fake_modules()
    saved = {k: sys.modules.get(k) for k in fakes}
    sys.modules.update(fakes)
    try:
        mod = types.ModuleType(name)
        mod.__file__ = path
        code = compile(src, path, 'exec')
        exec(code, mod.__dict__)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    _MODULE_CACHE[name] = mod
    return mod


@contextlib.contextmanager
def quiet():
    """Swallow the reference's progress prints."""
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        yield buf
