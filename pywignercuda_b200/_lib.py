"""ctypes binding of ``libwigner_b200.so`` (declared in include/wigner_b200.h).

The reference binds cuFFT the same way (``cufft_wrapper.py:78-145``) and maps
its status codes to exception classes (``cufft_wrapper.py:15-75``); this module
does the same for the propagators' C ABI.  There is no fallback: if the
library is missing the import of the propagator classes fails loudly.
"""
import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_uint32, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libwigner_b200.so')

ABI_VERSION = 4
WIG_NOBS = 11
WIG_BLOCH_NSTATS = 10
DIRAC_NOBS = 10
DIRAC3_NOBS = 12
WIG_RUN_CONTINUE = 1
WIG_RUN_PROFILE = 2
WIG_RUN_GRAPH = 4
WIG_RUN_FLUSH_L2 = 8

DAMP_NONE, DAMP_CALDEIRA_LEGGETT, DAMP_ODM = 0, 1, 2
CONST_CUDA_F, CONST_EXACT = 0, 1
PREC_C128 = 0
PREC_F32 = 1
PHASE_MOYAL, PHASE_KVN = 0, 1
SPLIT_LIE, SPLIT_STRANG_GP = 0, 1


class WignerError(RuntimeError):
    """Base class of the propagator library's errors."""


class WignerArgumentError(WignerError, ValueError):
    pass


class WignerCompileError(WignerError):
    pass


class WignerCudaError(WignerError):
    pass


class WignerTimeoutError(WignerError):
    pass


class WignerNonFiniteError(WignerError, FloatingPointError):
    pass


class WignerUnsupportedError(WignerError, NotImplementedError):
    pass


class WignerMemoryError(WignerError, MemoryError):
    pass


_EXC = {1: WignerArgumentError, 2: WignerCompileError, 3: WignerCudaError, 4: WignerTimeoutError,
        5: WignerNonFiniteError, 6: WignerUnsupportedError, 7: WignerMemoryError}

_DP = POINTER(c_double)


class WigDesc(ctypes.Structure):
    _fields_ = [('abi_version', c_int32), ('n_x', c_int32), ('n_p', c_int32), ('damping', c_int32),
                ('kinetic_from_string', c_int32), ('constants', c_int32), ('precision', c_int32),
                ('n_lindblad', c_int32), ('potential_phase', c_int32), ('skip_normalise', c_int32),
                ('splitting', c_int32), ('reserved0', c_int32),
                ('x_amplitude', c_double), ('p_amplitude', c_double), ('hbar', c_double),
                ('mass', c_double), ('dt', c_double), ('d_theta', c_double), ('d_lambda', c_double),
                ('gamma', c_double), ('epsilon', c_double), ('l_material', c_double),
                ('weight1', c_double), ('weight2', c_double), ('gp_coefficient', c_double),
                ('potential', c_char_p), ('kinetic', c_char_p), ('fp_damping', c_char_p), ('dpotential', c_char_p),
                ('x_table', _DP), ('p_table', _DP), ('theta_table', _DP), ('lambda_table', _DP),
                ('dv_table', _DP), ('v0_table', _DP), ('coef', c_double * 8)]


class WigbInstance(ctypes.Structure):
    _fields_ = [('n_x', c_int32), ('n_p', c_int32), ('damping_f', c_int32), ('reserved', c_int32),
                ('x_amplitude', c_double), ('p_amplitude', c_double), ('hbar', c_double), ('mass', c_double),
                ('dt', c_double), ('d_theta', c_double), ('d_lambda', c_double), ('gamma', c_double),
                ('f_eps', c_double), ('v4', c_double), ('v2', c_double), ('v1', c_double), ('v0', c_double)]


WIGA_PREC_C64 = 0
WIGA_PREC_C128 = 1


class WigaDesc(ctypes.Structure):
    _fields_ = [('abi_version', c_int32), ('n_x', c_int32), ('n_p', c_int32), ('precision', c_int32),
                ('x_amplitude', c_double), ('p_amplitude', c_double), ('hbar', c_double), ('mass', c_double),
                ('dt', c_double), ('d_theta', c_double), ('d_lambda', c_double),
                ('v4', c_double), ('v2', c_double), ('v0', c_double), ('gamma', c_double), ('f_eps', c_double)]


class DiracDesc(ctypes.Structure):
    _fields_ = [('abi_version', c_int32), ('n_x', c_int32), ('n_y', c_int32), ('constants', c_int32),
                ('precision', c_int32), ('reserved', c_int32),
                ('x_amplitude', c_double), ('y_amplitude', c_double), ('mass', c_double),
                ('c', c_double), ('hbar', c_double), ('dt', c_double),
                ('a0', c_char_p), ('a1', c_char_p), ('a2', c_char_p), ('a3', c_char_p),
                ('x_table', _DP), ('y_table', _DP), ('px_table', _DP), ('py_table', _DP),
                ('coef', c_double * 8)]


class Dirac3Desc(ctypes.Structure):
    _fields_ = [('abi_version', c_int32), ('n_x', c_int32), ('n_y', c_int32), ('n_z', c_int32),
                ('constants', c_int32), ('precision', c_int32),
                ('x_amplitude', c_double), ('y_amplitude', c_double), ('z_amplitude', c_double),
                ('mass', c_double), ('c', c_double), ('hbar', c_double), ('dt', c_double),
                ('a0', c_char_p), ('a1', c_char_p), ('a2', c_char_p), ('a3', c_char_p),
                ('coef', c_double * 8)]


# (name, restype, argtypes) of every symbol include/wigner_b200.h declares
SIGNATURES = [
    ('wig_create', c_int, [POINTER(WigDesc), POINTER(c_void_p)]),
    ('wig_run', c_int, [c_void_p, c_void_p, c_int64, c_int64, c_uint32, _DP, c_void_p]),
    ('wig_run_host', c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_uint32, _DP, c_void_p]),
    ('wig_run_many', c_int, [POINTER(c_void_p), POINTER(c_void_p), c_int64, c_int64, c_int64, c_uint32,
                             POINTER(_DP), c_void_p]),
    ('wig_profile', c_int, [c_void_p, _DP, POINTER(c_int64)]),
    ('wig_run_probability_square', c_int, [c_void_p, _DP, c_int64]),
    ('wig_bloch_stats', c_int, [c_void_p, c_void_p, c_int32, _DP, c_void_p]),
    ('wig_bloch_step', c_int, [c_void_p, c_void_p, c_int64, c_double, c_void_p, _DP, c_void_p]),
    ('wig_destroy', c_int, [c_void_p]),
    ('dirac_create', c_int, [POINTER(DiracDesc), POINTER(c_void_p)]),
    ('dirac_run', c_int, [c_void_p, c_void_p, c_int64, c_int64, _DP, c_void_p]),
    ('dirac_run_many', c_int, [POINTER(c_void_p), POINTER(c_void_p), c_int64, c_int64, c_int64,
                               POINTER(_DP), c_void_p]),
    ('dirac_run_host', c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, _DP, c_void_p]),
    ('dirac_destroy', c_int, [c_void_p]),
    ('dirac3_create', c_int, [POINTER(Dirac3Desc), POINTER(c_void_p)]),
    ('dirac3_run', c_int, [c_void_p, c_void_p, c_int64, c_int64, c_uint32, _DP, c_void_p]),
    ('dirac3_run_host', c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_uint32, _DP, c_void_p]),
    ('dirac3_destroy', c_int, [c_void_p]),
    ('dirac3_jit_check', c_int, [POINTER(Dirac3Desc), c_char_p, c_int64]),
    ('wig_jit_check', c_int, [POINTER(WigDesc), c_char_p, c_int64]),
    ('dirac_jit_check', c_int, [POINTER(DiracDesc), c_char_p, c_int64]),
    ('wigb_create', c_int, [c_void_p, c_int64, c_int32, c_int32, POINTER(c_void_p)]),
    ('wigb_offsets', c_int, [c_void_p, POINTER(c_int64)]),
    ('wigb_run', c_int, [c_void_p, c_void_p, c_int64, c_int64, c_uint32, _DP, c_void_p]),
    ('wigb_autotune', c_int, [c_void_p, c_void_p, c_int64, POINTER(c_int32), _DP, c_void_p]),
    ('wigb_profile', c_int, [c_void_p, _DP, POINTER(c_int64)]),
    ('wigb_destroy', c_int, [c_void_p]),
    ('wigb_jit_check', c_int, [POINTER(c_int32), c_int64, c_int32, c_int32, c_char_p, c_int64]),
    ('wiga_create', c_int, [POINTER(WigaDesc), POINTER(c_void_p)]),
    ('wiga_set_potential', c_int, [c_void_p, c_double, c_double, c_double]),
    ('wiga_forward', c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_void_p, c_void_p,
                             c_void_p]),
    ('wig_step_adjoint', c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_void_p,
                                 c_void_p]),
    ('wiga_adjoint_sweep', c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int64,
                                   c_void_p, c_void_p]),
    ('wiga_destroy', c_int, [c_void_p]),
    ('wiga_jit_check', c_int, [POINTER(WigaDesc), c_char_p, c_int64]),
    ('wig_observables_noalloc', c_int, [c_void_p, c_int32, c_int32, c_double, c_double, c_double, c_void_p,
                                        c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ('wig_last_error', c_char_p, []),
    ('wig_abi_version', c_int, []),
]

_lib = None


def load():
    """Load the native library (built by ``pywignercuda_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError('libwigner_b200.so is not built: run `python -m pywignercuda_b200.build` '
                              '(there is no CPU fallback)')
        lib = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        if lib.wig_abi_version() != ABI_VERSION:
            raise ImportError('libwigner_b200.so ABI %d, expected %d' % (lib.wig_abi_version(), ABI_VERSION))
        _lib = lib
    return _lib


def check(rc, what=''):
    if rc != 0:
        msg = load().wig_last_error().decode(errors='replace')
        raise _EXC.get(rc, WignerError)('%s failed (status %d): %s' % (what, rc, msg))


def dptr(a):
    """ctypes double* of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(_DP)
