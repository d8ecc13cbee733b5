"""The C-ABI library without a GPU: it loads, exports every symbol the header
declares, validates descriptors on the host, and its JIT source compiles with
NVRTC for sm_100a (compile only)."""
import ctypes
import os
import re

import pytest

from conftest import full_only
from pywignercuda_b200 import _lib
from pywignercuda_b200._lib import WigDesc, DiracDesc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, 'include', 'wigner_b200.h')).read()
    return sorted(set(re.findall(r'^\s*(?:int|const char\*)\s+(\w+)\s*\(', src, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 12
    for s in syms:
        assert hasattr(lib, s), s
    assert {n for n, _, _ in _lib.SIGNATURES} == set(syms)
    assert lib.wig_abi_version() == _lib.ABI_VERSION


def wig_desc(nx=256, npp=256, **kw):
    d = WigDesc()
    d.abi_version = _lib.ABI_VERSION
    d.n_x, d.n_p = nx, npp
    d.damping = kw.get('damping', _lib.DAMP_CALDEIRA_LEGGETT)
    d.x_amplitude = d.p_amplitude = 10.
    d.hbar = d.mass = 1.
    d.dt = 0.01
    d.gamma = kw.get('gamma', 0.1)
    d.d_theta = 0.1
    d.potential = kw.get('potential', b'0.05*pow(x,4) - pow(x,2)')
    d.kinetic = b'0.5*p*p'
    d.fp_damping = kw.get('fp', b'fabs(p)')
    return d


def jit(d, fn='wig_jit_check'):
    buf = ctypes.create_string_buffer(1 << 16)
    rc = getattr(_lib.load(), fn)(d, buf, len(buf))
    return rc, buf.value.decode()


@pytest.mark.parametrize('n', [16, 256, 1024, 4096])
def test_wigner_jit_compiles(n):
    rc, log = jit(wig_desc(n, n))
    assert rc == 0, log
    assert 'wig_xpass' in log and 'wig_ppass' in log
    assert '0 bytes spill stores' in log
    # the x-pass's register target follows the butterflies a thread holds per stage, so it
    # spills at most a few bytes at every size (the exact count depends on the NVRTC loaded)
    lines = log.splitlines()
    at = [i for i, l in enumerate(lines) if "Compiling entry function 'wig_xpass'" in l]
    props = ' '.join(lines[at[0] + 1:at[0] + 3])
    assert int(props.split(' bytes spill stores')[0].split()[-1]) <= 16, props


@pytest.mark.parametrize('n,tma', [(1024, '1'), (64, '0'), full_only(1024, '0'), full_only(64, '1')])
def test_register_fft_passes_compile(monkeypatch, n, tma):
    """The opt-in register-FFT passes (WIG_RF) compile under NVRTC, with the p-pass
    tile loaded by TMA or by the threads.  At 1024 points the p-pass holds 32 FP64 complex
    values a lane for each of its column pairs and spills a few hundred bytes (one reason
    the path stays opt-in); below that it spills at most a few bytes."""
    monkeypatch.setenv('WIG_RF', '1')
    monkeypatch.setenv('WIG_TMA', tma)
    rc, log = jit(wig_desc(n, n))
    assert rc == 0, log
    assert 'wig_xpass_rf' in log and 'wig_ppass_rf' in log
    lines = log.splitlines()
    for k in ('wig_xpass_rf', 'wig_ppass_rf'):
        at = [i for i, l in enumerate(lines) if "Compiling entry function '%s'" % k in l]
        props = ' '.join(lines[at[0] + 1:at[0] + 3])
        assert int(props.split(' bytes spill stores')[0].split()[-1]) <= (64 if n < 1024 else 512), (k, props)


def test_dirac_tiling_override_validated(monkeypatch):
    """WIG_DIRAC_TILING replaces the planner's tiles; a tile that does not divide
    the grid is refused on the host, before any compile."""
    d = DiracDesc()
    d.abi_version = _lib.ABI_VERSION
    d.n_x = d.n_y = 64
    d.x_amplitude = d.y_amplitude = 12.
    d.mass, d.c, d.hbar, d.dt = 1., 137.036, 1., 1e-4
    monkeypatch.setenv('WIG_DIRAC_TILING', '3,0,0,0,0,0')
    rc, log = jit(d, 'dirac_jit_check')
    assert rc == 1 and 'must divide the grid' in log      # WIG_ERR_ARG
    monkeypatch.setenv('WIG_DIRAC_TILING', '2,64,2,2,64,2')
    rc, log = jit(d, 'dirac_jit_check')
    assert rc == 0, log


@pytest.mark.parametrize('nx,ny', [(512, 512), (64, 32), (1024, 1024), (16, 2048)])
def test_dirac_jit_compiles(nx, ny):
    d = DiracDesc()
    d.abi_version = _lib.ABI_VERSION
    d.n_x, d.n_y = nx, ny
    d.x_amplitude = d.y_amplitude = 12.
    d.mass, d.c, d.hbar, d.dt = 1., 137.036, 1., 1e-4
    d.a0 = b'-1./sqrt(x*x+y*y+0.5)'
    d.a1 = b'-0.5*y'
    d.a2 = b'0.5*x'
    rc, log = jit(d, 'dirac_jit_check')
    assert rc == 0, log
    lines = log.splitlines()
    for k in ('dirac_rowpass', 'dirac_colpass'):
        at = [i for i, l in enumerate(lines) if "Compiling entry function '%s'" % k in l]
        assert at, k
        props = ' '.join(lines[at[0] + 1:at[0] + 3])
        spill = int(props.split(' bytes spill stores')[0].split()[-1])
        # up to 512-point axes the passes run 3 / 4 CTAs per SM (80 / 64 registers), 1024-point
        # axes 2: a few bytes may spill, how many depends on the NVRTC in the process (the
        # toolkit's, or the one torch loads first)
        assert spill <= 16, (k, props)


@pytest.mark.parametrize('nx,npp', [(100, 256), (256, 8), (8192, 256), (0, 0)])
def test_bad_grid_rejected_on_host(nx, npp):
    rc, log = jit(wig_desc(nx, npp))
    assert rc == 1 and 'powers of two' in log


def test_bad_expression_reports_compile_error():
    rc, log = jit(wig_desc(potential=b'0.5*pow(x,2) + undefined_name'))
    assert rc == 2 and 'undefined_name' in log


@pytest.mark.parametrize('expr', [b'x); } __global__ void k() { (x', b'x;', b'#define', b'((x)'])
def test_expression_injection_refused(expr):
    rc, log = jit(wig_desc(potential=expr))
    assert rc == 1


def test_kvn_phase_compiles_and_is_validated():
    d = wig_desc(256, 256)
    d.potential_phase = _lib.PHASE_KVN
    d.dpotential = b'0.2*pow(x,3) - 2.*x + 0.3*sin(3.*t)'
    rc, log = jit(d)
    assert rc == 0, log
    d.damping = _lib.DAMP_ODM
    d.l_material, d.n_lindblad = 1., 1
    rc, log = jit(d)
    assert rc == 6 and 'ODM' in log, log            # WIG_ERR_UNSUPPORTED
    d = wig_desc(256, 256)
    d.potential_phase = 7
    rc, log = jit(d)
    assert rc == 1 and 'potential_phase' in log, log
    d = wig_desc(256, 256)
    d.potential_phase = _lib.PHASE_KVN
    d.dpotential = b'x); }'
    rc, log = jit(d)
    assert rc == 1, log


def test_strang_gp_compiles_and_is_validated():
    d = wig_desc(256, 128)
    d.splitting = _lib.SPLIT_STRANG_GP
    d.kinetic_from_string = 1
    d.gp_coefficient = 0.5
    rc, log = jit(d)
    assert rc == 0, log
    for k in ('wig_ppass_half', 'wig_ppass_half_final', 'wig_gp_colsum', 'wig_gp_marginal', 'wig_gp_phase',
              'wig_bloch_ppass', 'wig_bloch_xpass', 'wig_gp_bloch', 'wig_bloch_reduce', 'wig_rowsum',
              'wig_bloch_axpy'):
        assert k in log, k
    d.potential_phase = _lib.PHASE_KVN
    rc, log = jit(d)
    assert rc == 6 and 'Strang' in log, log
    d = wig_desc(256, 128)
    d.gp_coefficient = 0.5                           # GP term without the Strang splitting
    rc, log = jit(d)
    assert rc == 1 and 'gp_coefficient' in log, log


def test_odm_kernels_compile():
    d = wig_desc(1024, 1024, damping=_lib.DAMP_ODM, fp=b' p*p/sqrt( p*p + 0.5 ) ')
    d.n_lindblad, d.l_material = 2, 3.
    rc, log = jit(d)
    assert rc == 0, log
    assert 'wig_odm_xpass' in log and 'wig_odm_ppass' in log


def test_python_classes_fail_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip('GPU present')
    from pywignercuda_b200 import GPU_Wigner2D_FFT, WignerCudaError

    class Inst(GPU_Wigner2D_FFT):
        def __init__(self):
            self.dampingFunction = 'CaldeiraLeggett'
            self.grossPitaevskiiCoefficient = 0.
            self.fp_Damping_String = 'fabs(p)'
            self.SetTimeTrack(0.01, 10, 100)
            GPU_Wigner2D_FFT.__init__(self, 256, 256, 10., 10., 1., 1., 0., 0., 0., '0.5*pow(x,2)', 'x',
                                      '0.5*p*p')
    with pytest.raises(WignerCudaError):
        Inst()


@pytest.mark.parametrize('precision,warps', [(0, 4), (1, 2), full_only(0, 8), full_only(0, 2), full_only(1, 8),
                                             full_only(1, 4)])
def test_batch_jit_spills_bounded(warps, precision):
    """All size classes in one kernel, at the default register caps (warps per SM:
    FP32 x-pass 16, p-pass 12; mixed 12 and 12; 8-warp tiles one CTA per SM).  The
    FP32 passes spill at most a few dozen bytes; the mixed p-pass at 168 registers
    spills ~1.1 KB (its 1024-point FP64 Moyal pair holds 32 double2 per lane), the
    trade that measured faster than 255 registers at 8 warps per SM."""
    sizes = (ctypes.c_int32 * 5)(64, 128, 256, 512, 1024)
    buf = ctypes.create_string_buffer(1 << 17)
    rc = _lib.load().wigb_jit_check(sizes, 5, warps, precision, buf, len(buf))
    log = buf.value.decode()
    assert rc == 0, log
    lines = log.splitlines()
    for k in ('wigb_xpass', 'wigb_ppass', 'wigb_reduce', 'wigb_scale'):
        at = [i for i, l in enumerate(lines) if "Compiling entry function '%s'" % k in l]
        assert at, k
        props = ' '.join(lines[at[0] + 1:at[0] + 3])
        spill = int(props.split(' bytes spill stores')[0].split()[-1])
        assert spill <= (32 if precision == 0 else 1536), (k, props)


def test_batch_precision_validated():
    sizes = (ctypes.c_int32 * 1)(128)
    buf = ctypes.create_string_buffer(4096)
    assert _lib.load().wigb_jit_check(sizes, 1, 4, 2, buf, len(buf)) == 1


def d3_desc(nx=64, ny=32, nz=128, **kw):
    from pywignercuda_b200._lib import Dirac3Desc
    d = Dirac3Desc()
    d.abi_version = _lib.ABI_VERSION
    d.n_x, d.n_y, d.n_z = nx, ny, nz
    d.constants = _lib.CONST_CUDA_F
    d.precision = _lib.PREC_C128
    d.x_amplitude = d.y_amplitude = d.z_amplitude = 8.
    d.mass, d.c, d.hbar, d.dt = kw.get('mass', 1.), 137.036, 1., 1e-4
    d.a0 = kw.get('a0', b'-1./sqrt(x*x+y*y+z*z+0.5)')
    d.a1 = b'-0.5*y'
    d.a2 = b'0.5*x'
    d.a3 = b'0.'
    return d


@pytest.mark.parametrize('shape', [(64, 32, 128), (256, 256, 256), (512, 16, 512)])
def test_dirac3d_jit_compiles_without_spills(shape):
    rc, log = jit(d3_desc(*shape), 'dirac3_jit_check')
    assert rc == 0, log
    lines = log.splitlines()
    for k in ('d3_xpass', 'd3_ypass_fwd', 'd3_ypass_inv', 'd3_zpass', 'd3_norm', 'd3_norm_fin'):
        at = [i for i, l in enumerate(lines) if "Compiling entry function '%s'" % k in l]
        assert at, k
        props = ' '.join(lines[at[0] + 1:at[0] + 3])
        spill = int(props.split(' bytes spill stores')[0].split()[-1])
        # the z- and x-passes run two and three CTAs per SM (128 / 80 registers): a few bytes may spill
        assert spill <= {'d3_zpass': 128, 'd3_xpass': 16}.get(k, 0), (k, props)


def test_dirac3d_descriptor_validated():
    rc, log = jit(d3_desc(48, 32, 32), 'dirac3_jit_check')
    assert rc == 1 and 'power of two' in log
    rc, log = jit(d3_desc(32, 32, 1024), 'dirac3_jit_check')
    assert rc == 1 and 'power of two' in log
    rc, log = jit(d3_desc(mass=0.), 'dirac3_jit_check')
    assert rc == 1 and 'mass' in log
    rc, log = jit(d3_desc(a0=b'x); }'), 'dirac3_jit_check')
    assert rc == 1 and 'expression' in log
    rc, log = jit(d3_desc(a0=b'unknown_name(x)'), 'dirac3_jit_check')
    assert rc != 0


def _wigb(n_x=128, n_p=128, **kw):
    d = _lib.WigbInstance()
    d.n_x, d.n_p = n_x, n_p
    d.x_amplitude = d.p_amplitude = 10.
    d.hbar = d.mass = 1.
    d.dt = 0.005
    for k, v in kw.items():
        setattr(d, k, v)
    return d


@pytest.mark.parametrize('bad,msg', [
    (dict(count=0), 'empty batch'),
    (dict(n_x=32), 'powers of two in [64, 1024]'),
    (dict(n_p=2048), 'powers of two in [64, 1024]'),
    (dict(n_x=96), 'powers of two in [64, 1024]'),
    (dict(x_amplitude=0.), 'amplitudes > 0'),
    (dict(mass=0.), 'hbar and mass nonzero'),
    (dict(dt=float('nan')), 'dt finite'),
    (dict(damping_f=2), 'damping_f'),
    (dict(warps=3), 'warps must be'),
    (dict(precision=5), 'precision must be'),
])
def test_batch_descriptors_validated_on_host(bad, msg):
    """wigb_create refuses an empty batch, grids outside the batched range (powers
    of two in [64, 1024], ragged n_x != n_p allowed), degenerate constants, an
    unknown damping function, tile shape or precision with WIG_ERR_ARG and a
    message, before touching the GPU; the second instance of a batch is checked
    like the first."""
    bad = dict(bad)
    count, warps, precision = bad.pop('count', 2), bad.pop('warps', 0), bad.pop('precision', 0)
    second = dict(n_x=256, n_p=64)
    second.update(bad)
    arr = (_lib.WigbInstance * 2)(_wigb(), _wigb(**second))
    h = ctypes.c_void_p()
    rc = _lib.load().wigb_create(ctypes.cast(arr, ctypes.c_void_p), count, warps, precision, ctypes.byref(h))
    assert rc == 1 and not h.value
    assert msg in _lib.load().wig_last_error().decode(), _lib.load().wig_last_error()


@pytest.mark.parametrize('field,value', [('n_x', 48), ('n_p', 4096), ('precision', 2), ('abi_version', 3),
                                         ('x_amplitude', -1.), ('gamma', float('inf')), ('f_eps', -1.)])
def test_adjoint_descriptor_validated_on_host(field, value):
    d = _lib.WigaDesc()
    d.abi_version = _lib.ABI_VERSION
    d.n_x = d.n_p = 128
    d.precision = _lib.WIGA_PREC_C128
    d.x_amplitude = d.p_amplitude = 10.
    d.hbar = d.mass = 1.
    d.dt = 0.005
    setattr(d, field, value)
    h = ctypes.c_void_p()
    assert _lib.load().wiga_create(ctypes.byref(d), ctypes.byref(h)) == 1
    assert not h.value


def _batch_regs(precision, warps=2, sizes=(1024,)):
    arr = (ctypes.c_int32 * len(sizes))(*sizes)
    buf = ctypes.create_string_buffer(1 << 17)
    assert _lib.load().wigb_jit_check(arr, len(sizes), warps, precision, buf, len(buf)) == 0, buf.value
    lines = buf.value.decode().splitlines()
    out = {}
    for k in ('wigb_xpass', 'wigb_ppass'):
        at = [i for i, l in enumerate(lines) if "Compiling entry function '%s'" % k in l][0]
        out[k] = int(re.search(r'Used (\d+) registers', ' '.join(lines[at + 1:at + 4])).group(1))
    return out


def test_batch_register_caps_and_override(monkeypatch):
    """The batched passes' default register caps (FP32 x-pass: 16 warps per SM, so at
    most 128 registers a thread in a 2-warp tile; p-pass: 12, 168) and the
    WIG_BATCH_WPS=x,p override, which recompiles them for other warps-per-SM targets."""
    regs = _batch_regs(0)
    assert regs['wigb_xpass'] <= 128 and regs['wigb_ppass'] <= 168, regs
    monkeypatch.setenv('WIG_BATCH_WPS', '8,8')
    regs = _batch_regs(0)
    assert regs['wigb_xpass'] > 128 and regs['wigb_ppass'] > 168, regs


def test_adjoint_sweep_arguments_validated_on_host():
    """wiga_adjoint_sweep refuses an empty segment and a missing handle before any
    launch (WIG_ERR_ARG)."""
    lib = _lib.load()
    buf = ctypes.create_string_buffer(64)
    p = ctypes.cast(buf, ctypes.c_void_p)
    assert lib.wiga_adjoint_sweep(None, p, p, None, None, p, 0, 0, p, None) == 1
    assert 'n_steps' in lib.wig_last_error().decode()
    assert lib.wiga_adjoint_sweep(None, p, p, None, None, p, 0, 4, p, None) == 1
    assert 'null handle' in lib.wig_last_error().decode()
