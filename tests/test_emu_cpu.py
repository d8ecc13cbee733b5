"""The complex128 Wigner2D, Dirac2D and Dirac3D kernels' device code, executed
on the host (tests/emu/shim.h: one thread per CUDA thread, real barriers and
shuffles), against the oracle.

It checks the passes' tiling, index arithmetic, partial-sum reductions and the
launch sequences of wig_run, dirac_run and dirac3_run, for the tile shapes the
planners pick at large grids and others, without a GPU.  The device sources
are the ones NVRTC compiles for sm_100a; only `extern __shared__` arrays are
pointed at a host buffer."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import full_only
from oracle.common import rel_l2
from oracle.dirac2d import DiracOracle, DiracParams, spinor_particle_spin_up
from oracle.dirac3d import Dirac3DOracle, Dirac3DParams, spinor_particle_spin_up_3d
from oracle.wigner2d import WignerOracle, WignerParams, wigner_harmonic_oscillator
from batch_cases import random_batch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, 'pywignercuda_b200', 'csrc')
EMU = os.path.join(ROOT, 'tests', 'emu')
HEADERS = ('wig_fft.cuh', 'wig_wigner.cuh', 'wig_dirac.cuh', 'wig_jit_dirac.cuh', 'wig_jit_wigner.cuh',
           'wig_dirac3.cuh', 'wig_jit_dirac3.cuh', 'wig_rfft.cuh', 'wig_batch.cuh', 'wig_jit_batch.cuh',
           'wig_adjoint.cuh', 'wig_jit_adjoint.cuh', 'wig_batch_host.h', 'wig_adjoint_host.h', 'wig_wigner_rf.cuh')
EXTERN_SHARED = re.compile(r'extern\s+__shared__\s+(\w+)\s+(\w+)\s*\[\s*\]\s*;')

NX, NY = 32, 16
XA, YA, DT, MASS, C = 12., 8., 1e-3, 1., 137.036
A = ('-1./sqrt(x*x+y*y+0.5) + 0.3*t*x', '-0.5*y', '0.5*x', '0.')   # as in tests/emu/dirac2d_emu.cpp


def stage(dst):
    for h in HEADERS:
        src = open(os.path.join(CSRC, h)).read()
        src = EXTERN_SHARED.sub(lambda m: '%s* %s = reinterpret_cast<%s*>(emu_smem);'
                                % (m.group(1), m.group(2), m.group(1)), src)
        open(os.path.join(dst, h), 'w').write(src)
    for f in ('shim.h', 'dirac2d_emu.cpp', 'wigner2d_emu.cpp', 'dirac3d_emu.cpp', 'batch_emu.cpp', 'adjoint_emu.cpp',
              'round_emu.cpp'):
        shutil.copy(os.path.join(EMU, f), dst)


SANITIZE = {None: [], 'thread': ['-fsanitize=thread', '-g'], 'address': ['-fsanitize=address,undefined', '-g',
                                                                       '-fno-sanitize-recover=undefined']}


def build(dst, source, macros, sanitize=None):
    """g++ build of an emulation driver, with the device code's index checks
    (WIG_BOUNDS) on; sanitize: None, 'thread' (data races, including shared-memory
    accesses not ordered by a barrier) or 'address' (address + undefined behaviour:
    accesses past a launch's exact dynamic shared memory, heap overflows)."""
    tag = ''.join('_%s' % re.sub(r'\W', '', str(v)) for v in macros.values()) + ('_' + sanitize if sanitize else '')
    exe = os.path.join(dst, source.split('.')[0] + tag)
    cmd = (['g++', '-std=c++20', '-O1', '-pthread', '-w', '-DWIG_BOUNDS', '-I', dst] + SANITIZE[sanitize] +
           ['-D%s=%s' % kv for kv in macros.items()] + [os.path.join(dst, source), '-o', exe])
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


@pytest.fixture(scope='module')
def staged(tmp_path_factory):
    if shutil.which('g++') is None:
        pytest.skip('no host C++ compiler')
    d = str(tmp_path_factory.mktemp('emu'))
    stage(d)
    return d


# (rows, row threads, columns, column threads) per CTA: the planner's rule at 32 x 16 (one CTA per
# pass), several CTAs per pass, and one row / one column per CTA as at 512^2
@pytest.mark.parametrize('rows,rnt,cc,cnt', [(16, 256, 32, 256), full_only(4, 64, 8, 64), (1, 32, 1, 32)])
def test_dirac2d_device_code_matches_oracle(staged, rows, rnt, cc, cnt):
    exe = build(staged, 'dirac2d_emu.cpp', dict(DIR_NX=NX, DIR_NY=NY, DIR_ROWS=rows, DIR_RNT=rnt, DIR_RMB=1,
                                                DIR_C=cc, DIR_CNT=cnt, DIR_CMB=1, DIR_SNT=256))
    prm = DiracParams(NX, NY, XA, YA, DT, mass=MASS, c=C, A0=A[0], A1=A[1], A2=A[2], A3=A[3],
                      constants='exact')
    psi0 = spinor_particle_spin_up(prm, (2., 1.), lambda x, y: np.exp(-(x * x + y * y) / 4.))
    psi0 = np.ascontiguousarray(psi0, dtype=np.complex128)
    steps = 2      # the first, a continuing and the last launch of each kind
    fin, fout, fobs = (os.path.join(staged, n) for n in ('psi_in.bin', 'psi_out.bin', 'obs.bin'))
    psi0.tofile(fin)
    r = subprocess.run([exe, fin, fout, fobs, str(steps), repr(XA), repr(YA), repr(DT), repr(MASS), repr(C)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = np.fromfile(fout, dtype=np.complex128).reshape(4, NY, NX)
    obs = np.fromfile(fobs).reshape(steps, 10)
    ref_obs, ref = DiracOracle(prm).run(psi0, steps)
    assert rel_l2(got, ref) < 1e-12
    scale = np.maximum(np.abs(ref_obs).max(axis=0), 1e-3)
    assert np.all(np.abs(obs - ref_obs) / scale < 1e-10), (obs - ref_obs) / scale


WNX, WNP = 64, 32
WXA, WPA, WDT, WGAMMA, WDTH, WDLA = 10., 8., 0.01, 0.1, 0.1, 0.05
# as in tests/emu/wigner2d_emu.cpp
WPOT, WDPOT = '0.05*pow(x,4) - pow(x,2) + 0.2*x*sin(3.*t)', '0.2*pow(x,3) - 2.*x + 0.2*sin(3.*t)'


# (rows, x threads, columns, p threads) per CTA: the planner's rule at 64 x 32 (one CTA per pass),
# one row per 128-thread CTA as for 1024-point rows, and several small CTAs per pass; Caldeira-Leggett,
# ODM Lindblad damping (first order) on two of the shapes, GPU_Wigner2D_ODM2 (damping and pumping terms,
# kinetic factor from the kinetic string), and the Fokker-Planck (KvN) potential factor
@pytest.mark.parametrize('xrows,xnt,pc,pnt,odm,kvn', [(32, 256, 64, 256, 0, 0), (1, 128, 2, 32, 0, 0),
                                                      (4, 32, 8, 32, 0, 0), (32, 256, 64, 256, 1, 0),
                                                      (4, 32, 8, 32, 1, 0), (4, 32, 8, 32, 2, 0),
                                                      (4, 32, 8, 32, 0, 1)])
def test_wigner2d_device_code_matches_oracle(staged, xrows, xnt, pc, pnt, odm, kvn):
    exe = build(staged, 'wigner2d_emu.cpp', dict(WIG_NX=WNX, WIG_NP=WNP, WIG_XROWS=xrows, WIG_XNT=xnt,
                                                 WIG_KIN_STRING=int(odm == 2), WIG_PC=pc, WIG_PNT=pnt,
                                                 WIG_DAMP=int(odm == 0), WIG_RNT=256, WIG_XMINB=1, WIG_PMINB=1,
                                                 WIG_KVN=kvn))
    prm = WignerParams(WNX, WNP, WXA, WPA, WDT, d_theta=WDTH, d_lambda=WDLA, gamma=WGAMMA, potential=WPOT,
                       dpotential=WDPOT, kinetic='0.5*p*p', damping='ODM' if odm else 'CaldeiraLeggett',
                       fp_damping='fabs(p)', L_material=1., kvn=bool(kvn), odm2=odm == 2, weight1=1.,
                       weight2=0.5 if odm == 2 else 0., constants='exact')
    X = np.fft.fftshift(np.linspace(-WXA, WXA - 2 * WXA / WNX, WNX))[np.newaxis, :]
    P = np.fft.fftshift(np.linspace(-WPA, WPA - 2 * WPA / WNP, WNP))[:, np.newaxis]
    W0 = np.ascontiguousarray(np.exp(-(X - 1.5) ** 2 - (P + 0.5) ** 2 * 1.3) + 0. * 1j)
    steps = 2      # the first, a continuing and the last launch of each kind
    fin, fout, fobs = (os.path.join(staged, n) for n in ('w_in.bin', 'w_out.bin', 'w_obs.bin'))
    W0.tofile(fin)
    r = subprocess.run([exe, fin, fout, fobs, str(steps)] + [repr(v) for v in (WXA, WPA, WDT, WGAMMA, WDTH, WDLA)] +
                       [str(odm), '0.'], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = np.fromfile(fout, dtype=np.complex128).reshape(WNP, WNX)
    obs = np.fromfile(fobs).reshape(steps + 1, 11)
    ref_obs, ref = WignerOracle(prm).run(W0, steps)
    assert rel_l2(got, ref) < 1e-12
    scale = np.maximum(np.abs(ref_obs[:, :10]).max(axis=0), 1e-3)
    assert np.all(np.abs(obs[:, :10] - ref_obs[:, :10]) / scale < 1e-10), (obs[:, :10] - ref_obs[:, :10]) / scale
    # the negative area (here ~ -4e-5) sums the points below zero: points within rounding of zero
    # enter one sum and not the other, so it is held to an absolute 1e-12
    assert np.all(np.abs(obs[:, 10] - ref_obs[:, 10]) < 1e-12), obs[:, 10] - ref_obs[:, 10]


# The register-FFT x- and p-pass of Lie plans (wig_wigner_rf.cuh) on a 128 x 64 grid: Caldeira-Leggett,
# undamped, the Fokker-Planck (KvN) factor; one and several warps per CTA
@pytest.mark.parametrize('xw,pw,kvn,gamma', [(4, 2, 0, WGAMMA), full_only(1, 1, 0, WGAMMA), full_only(2, 2, 0, 0.),
                                              (4, 1, 1, WGAMMA)])
def test_wigner2d_rf_device_code_matches_oracle(staged, xw, pw, kvn, gamma):
    nx, npp = 128, 64
    damp = int(gamma != 0.)
    exe = build(staged, 'wigner2d_emu.cpp', dict(WIG_NX=nx, WIG_NP=npp, WIG_XROWS=1, WIG_XNT=32, WIG_KIN_STRING=0,
                                                 WIG_PC=2, WIG_PNT=32, WIG_DAMP=damp, WIG_RNT=256, WIG_XMINB=1,
                                                 WIG_PMINB=1, WIG_KVN=kvn, WIG_RF=1, WIG_RFXW=xw, WIG_RFPW=pw,
                                                 WIG_RFXMB=1, WIG_RFPMB=1))
    prm = WignerParams(nx, npp, WXA, WPA, WDT, d_theta=WDTH, d_lambda=WDLA, gamma=gamma, potential=WPOT,
                       dpotential=WDPOT, kinetic='0.5*p*p', damping='CaldeiraLeggett', fp_damping='fabs(p)',
                       kvn=bool(kvn), constants='exact')
    X = np.fft.fftshift(np.linspace(-WXA, WXA - 2 * WXA / nx, nx))[np.newaxis, :]
    P = np.fft.fftshift(np.linspace(-WPA, WPA - 2 * WPA / npp, npp))[:, np.newaxis]
    W0 = np.ascontiguousarray(np.exp(-(X - 1.5) ** 2 - (P + 0.5) ** 2 * 1.3) + 0. * 1j)
    steps = 2
    fin, fout, fobs = (os.path.join(staged, n) for n in ('wr_in.bin', 'wr_out.bin', 'wr_obs.bin'))
    W0.tofile(fin)
    r = subprocess.run([exe, fin, fout, fobs, str(steps)] + [repr(v) for v in (WXA, WPA, WDT, gamma, WDTH, WDLA)] +
                       ['0', '0.'], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = np.fromfile(fout, dtype=np.complex128).reshape(npp, nx)
    obs = np.fromfile(fobs).reshape(steps + 1, 11)
    ref_obs, ref = WignerOracle(prm).run(W0, steps)
    assert rel_l2(got, ref) < 1e-12, rel_l2(got, ref)
    scale = np.maximum(np.abs(ref_obs[:, :10]).max(axis=0), 1e-3)
    assert np.all(np.abs(obs[:, :10] - ref_obs[:, :10]) / scale < 1e-10), (obs[:, :10] - ref_obs[:, :10]) / scale
    assert np.all(np.abs(obs[:, 10] - ref_obs[:, 10]) < 1e-12), obs[:, 10] - ref_obs[:, 10]


# Strang splitting with the Gross-Pitaevskii mean-field term (GPU_Wigner2D_GPitaevskii): with
# Caldeira-Leggett, and with ODM damping on the planner's tile and on small CTAs
@pytest.mark.parametrize('xrows,xnt,pc,pnt,odm,a_gp', [(32, 256, 64, 256, 0, 0.5), (32, 256, 64, 256, 1, -0.3),
                                                       (4, 32, 8, 32, 1, -0.3)])
def test_strang_gp_device_code_matches_oracle(staged, xrows, xnt, pc, pnt, odm, a_gp):
    from oracle.gpitaevskii import GPitaevskiiOracle
    exe = build(staged, 'wigner2d_emu.cpp', dict(WIG_NX=WNX, WIG_NP=WNP, WIG_XROWS=xrows, WIG_XNT=xnt,
                                                 WIG_KIN_STRING=1, WIG_PC=pc, WIG_PNT=pnt, WIG_DAMP=1 - odm,
                                                 WIG_RNT=256, WIG_XMINB=1, WIG_PMINB=1, WIG_STRANG=1))
    prm = WignerParams(WNX, WNP, WXA, WPA, WDT, d_theta=WDTH, d_lambda=WDLA, gamma=WGAMMA, potential=WPOT,
                       dpotential=WDPOT, kinetic='0.5*p*p', damping='ODM' if odm else 'CaldeiraLeggett',
                       fp_damping='fabs(p)', L_material=1., constants='exact')
    X = np.fft.fftshift(np.linspace(-WXA, WXA - 2 * WXA / WNX, WNX))[np.newaxis, :]
    P = np.fft.fftshift(np.linspace(-WPA, WPA - 2 * WPA / WNP, WNP))[:, np.newaxis]
    W0 = np.ascontiguousarray(np.exp(-(X - 1.5) ** 2 - (P + 0.5) ** 2 * 1.3) + 0. * 1j)
    steps = 2      # the first, a continuing and the last launch of each kind
    fin, fout, fobs = (os.path.join(staged, n) for n in ('g_in.bin', 'g_out.bin', 'g_obs.bin'))
    W0.tofile(fin)
    r = subprocess.run([exe, fin, fout, fobs, str(steps)] + [repr(v) for v in (WXA, WPA, WDT, WGAMMA, WDTH, WDLA)] +
                       [str(odm), repr(a_gp)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = np.fromfile(fout, dtype=np.complex128).reshape(WNP, WNX)
    raw = np.fromfile(fobs)
    obs, psq = raw[:(steps + 1) * 11].reshape(steps + 1, 11), raw[(steps + 1) * 11:]
    ref_obs, ref, ref_psq = GPitaevskiiOracle(prm, a_gp).run(W0, steps)
    assert rel_l2(got, ref) < 1e-12
    # row 0 is the initial state's sample, row n + 1 the state after step n (the oracle's row n)
    scale = np.maximum(np.abs(ref_obs[:, :10]).max(axis=0), 1e-3)
    assert np.all(np.abs(obs[1:, :10] - ref_obs[:, :10]) / scale < 1e-10), (obs[1:, :10] - ref_obs[:, :10]) / scale
    assert np.all(np.abs(obs[1:, 10] - ref_obs[:, 10]) < 1e-12)
    assert np.max(np.abs(psq - ref_psq) / np.abs(ref_psq)) < 1e-10


D3 = (32, 16, 16)
D3A, D3DT = (10., 8., 8.), 1e-3
# as in tests/emu/dirac3d_emu.cpp
D3POT = ('-1./sqrt(x*x+y*y+z*z+0.5) + 0.2*t*z', '-0.5*y', '0.5*x', '0.1*z')


def d3_threads(n):
    return max(32, min(256, n)) // 32 * 32


# (rows, yc, zc, radix x / y / z, CTA cap): the planner's tiles at 32 x 16 x 16 (radix 16 on z),
# small tiles with every pass grid-striding over 5 CTAs, and radix 16 on every axis over 3 CTAs
@pytest.mark.parametrize('rows,yc,zc,xr,yr,zr,cap', [full_only(16, 32, 32, 8, 8, 16, 2368),
                                                     full_only(2, 4, 2, 8, 8, 16, 5), (16, 32, 32, 16, 16, 16, 3)])
def test_dirac3d_device_code_matches_oracle(staged, rows, yc, zc, xr, yr, zr, cap):
    _dirac3d_run(staged, D3, rows, yc, zc, xr, yr, zr, cap)


@pytest.mark.parametrize('n', [16, full_only(32)])
def test_dirac3d_cubic_planner_tiles(staged, n):
    """Cubic grids with the planner's tiles (dirac3_plan: rows = 512 / n, yc = 2048 / n and
    zc = 1024 / n clamped to n, radix 16 on z): the shapes at which the z-pass's K mix read
    stale spectra on the GPU without its explicit barrier."""
    _dirac3d_run(staged, (n, n, n), min(512 // n, n * n), min(max(2048 // n, 2), n), min(1024 // n, n), 8, 8, 16,
                 2368)


def _dirac3d_run(staged, dims, rows, yc, zc, xr, yr, zr, cap):
    nx, ny, nz = dims
    exe = build(staged, 'dirac3d_emu.cpp', dict(D3_NX=nx, D3_NY=ny, D3_NZ=nz, D3_ROWS=rows,
                                                D3_XNT=d3_threads(4 * rows * nx // 8), D3_YC=yc,
                                                D3_YNT=d3_threads(ny * yc // 8), D3_ZC=zc,
                                                D3_ZNT=d3_threads(4 * zc * nz // 8), D3_SNT=256, D3_XR=xr,
                                                D3_YR=yr, D3_ZR=zr, D3_XMB=1, D3_YMB=1, D3_ZMB=1))
    prm = Dirac3DParams(nx, ny, nz, *D3A, D3DT, mass=1., c=137.036, A0=D3POT[0], A1=D3POT[1], A2=D3POT[2],
                        A3=D3POT[3], constants='exact')
    psi0 = spinor_particle_spin_up_3d(prm, (2., 0.5, 1.), lambda x, y, z: np.exp(-(x * x + y * y + z * z) / 4.))
    psi0 = np.ascontiguousarray(psi0, dtype=np.complex128)
    steps = 2      # the first, a continuing and the last launch of each kind
    fin, fout, fobs = (os.path.join(staged, n) for n in ('p3_in.bin', 'p3_out.bin', 'p3_obs.bin'))
    psi0.tofile(fin)
    r = subprocess.run([exe, fin, fout, fobs, str(steps)] + [repr(v) for v in D3A + (D3DT, 1., 137.036)] +
                       [str(cap)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    got = np.fromfile(fout, dtype=np.complex128).reshape(4, nz, ny, nx)
    obs = np.fromfile(fobs).reshape(steps, 12)
    ref_obs, ref = Dirac3DOracle(prm).run(psi0, steps)
    assert rel_l2(got, ref) < 1e-12
    scale = np.maximum(np.abs(ref_obs).max(axis=0), 1e-3)
    assert np.all(np.abs(obs - ref_obs) / scale < 1e-10), (obs - ref_obs) / scale


@pytest.mark.parametrize('mode', ['seeds', 'stream'])
def test_stochastic_rounding_is_unbiased(staged, mode):
    """The mixed form's FP64 -> FP32 store (store_round over a lane's SrStream
    seeded by sr_word / sr_key): each result is one of the two FP32 values
    bracketing v (v itself when it is one), rounds away from zero with
    probability equal to v's fraction of the ulp -- so the mean over steps
    converges to v -- and non-finite values stay non-finite.  The words are the
    first word of each step's stream ('seeds': what one point sees over steps) or
    the consecutive words of one stream ('stream': what one lane's points see in
    one step).  Also: one value stored at many lanes' first points in one step
    rounds up at the same rate (the seeds are uncorrelated across elements)."""
    exe = build(staged, 'round_emu.cpp', {'WIGB_WARPS': 4, 'WIGB_PREC': 1, 'WIGB_CASES(F)': 'F(64)'})
    rng = np.random.default_rng(3)
    mags = np.exp(rng.uniform(np.log(1e-30), np.log(1e3), 200)) * rng.choice([-1., 1.], 200)
    f32 = rng.standard_normal(20).astype(np.float32).astype(np.float64)          # already FP32
    lo = np.float32(0.7).astype(np.float64)
    ulp = np.nextafter(np.float32(0.7), np.float32(1.)).astype(np.float64) - lo
    fracs = lo + ulp * np.array([0.5, 0.25, 0.75, 0.01, 0.99])                   # known fractions
    vals = np.concatenate([mags, f32, fracs, -fracs, [0., -0., np.nan, np.inf, -np.inf]])
    steps = 4000
    fin, fout = os.path.join(staged, 'sr_in.bin'), os.path.join(staged, 'sr_out.bin')
    vals.tofile(fin)
    r = subprocess.run([exe, fin, fout, str(steps), '123456789', mode], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = np.fromfile(fout, dtype=np.float32).reshape(len(vals), steps).astype(np.float64)
    for v, o in zip(vals, out):
        if not np.isfinite(v):
            assert not np.isfinite(o).any(), v
            continue
        a = np.float32(v)                                   # nearest
        a = a.astype(np.float64)
        if a == v:
            assert np.all(o == v), v
            continue
        b = np.nextafter(np.float32(v), np.float32(np.inf if v > a else -np.inf)).astype(np.float64)
        lo_v, hi_v = (a, b) if abs(a) < abs(b) else (b, a)  # toward / away from zero
        assert np.all((o == lo_v) | (o == hi_v)), v
        p = (abs(v) - abs(lo_v)) / abs(hi_v - lo_v)
        up = np.mean(o == hi_v)
        assert abs(up - p) <= 5. * np.sqrt(max(p * (1. - p), 1e-3) / steps) + 2. ** -29, (v, p, up)
    # one step, one value at many elements
    vals = np.full(20000, lo + 0.5 * ulp)
    vals.tofile(fin)
    r = subprocess.run([exe, fin, fout, '1', '0', 'seeds'], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = np.fromfile(fout, dtype=np.float32).astype(np.float64)
    assert abs(np.mean(out > lo) - 0.5) < 5. * np.sqrt(0.25 / len(out))


# instances of the batched FP32 form: mixed grids, two of them non-square with unequal amplitudes,
# one undamped; one with the p^2 / sqrt(p^2 + eps) damping function, a lambda diffusion and linear and
# constant potential terms, another with a linear term
BSIZES = (64, 128, 128, 64)
BSHAPES = ((64, 128, 10., 8.), (128, 64, 8., 10.))
BEXTRA = {1: dict(ff=1, f_eps=0.5, d_lambda=0.01, v1=0.3, v0=0.2), 4: dict(v1=-0.2)}


@pytest.mark.parametrize('warps,grid,prec,xstage', [full_only(4, 3, 0, 0), (2, 5, 0, 1), (4, 3, 1, 0),
                                                     full_only(2, 5, 1, 1)])
def test_batch_device_code_matches_oracle(staged, warps, grid, prec, xstage):
    """The real-storage passes (two rows / columns per complex transform, the
    Nyquist split), in FP32 (prec 0) and with the FP64 kinetic and Moyal pairs
    and their in-place mirror split (prec 1; the 64-point grids with the FP64
    dissipator, the 128-point ones with the FP32 one), the persistent work lists
    and the last-CTA normalisation, against the FP64 oracle, 2 steps (each
    emulated step costs seconds of barrier traffic).  xstage 1: the x-pass rows arrive
    through the shared-memory staging buffer, one item ahead."""
    exe = build(staged, 'batch_emu.cpp', {'WIGB_WARPS': warps, 'WIGB_XMINB': 1, 'WIGB_PMINB': 1, 'WIGB_PREC': prec,
                                          'WIGB_XSTAGE': xstage, 'WIGB_DISS64_MAXN': 64,
                                          'WIGB_CASES(F)': 'F(64) F(128)'})
    cases = random_batch(list(BSIZES) + [s[0] for s in BSHAPES], seed=11)
    cases[2]['gamma'] = 0.
    for c, (nx, npp, xa, pa) in zip(cases[len(BSIZES):], BSHAPES):
        c.update(n_x=nx, n_p=npp, xa=xa, pa=pa)
    for i, extra in BEXTRA.items():
        cases[i].update(extra)
    steps, dt = 2, 0.005

    def g(c, k, d=0.):
        return c.get(k, d)

    def shape(c):
        return g(c, 'n_x', c['n']), g(c, 'n_p', c['n']), g(c, 'xa', 10.), g(c, 'pa', 10.)
    prm = np.array([[shape(c)[0], shape(c)[1], c['a'], c['b'], g(c, 'v1'), g(c, 'v0'), c['gamma'], c['gamma'],
                     g(c, 'd_lambda'), dt, shape(c)[2], shape(c)[3], g(c, 'ff'), g(c, 'f_eps', 0.5)]
                    for c in cases], dtype=np.float64)

    def params(c):
        nx, npp, xa, pa = shape(c)
        pot = '%r*pow(x,4) + %r*pow(x,2) + %r*x + %r' % (c['a'], c['b'], g(c, 'v1'), g(c, 'v0'))
        dpot = '4*%r*pow(x,3) + 2*%r*x + %r' % (c['a'], c['b'], g(c, 'v1'))
        f = 'fabs(p)' if not g(c, 'ff') else 'p*p/sqrt(p*p + %r)' % g(c, 'f_eps', 0.5)
        return WignerParams(nx, npp, xa, pa, dt, potential=pot, dpotential=dpot, gamma=c['gamma'],
                            d_theta=c['gamma'], d_lambda=g(c, 'd_lambda'), damping='CaldeiraLeggett',
                            fp_damping=f, constants='exact')
    W0 = [np.ascontiguousarray(wigner_harmonic_oscillator(params(c), 0, 1., c['x0'], c['p0'])) for c in cases]
    packed = np.concatenate([w.real.astype(np.float32).ravel() for w in W0])
    fprm, fin, fout, fobs = (os.path.join(staged, n) for n in ('b_prm.bin', 'b_in.bin', 'b_out.bin', 'b_obs.bin'))
    prm.tofile(fprm)
    packed.tofile(fin)
    r = subprocess.run([exe, fprm, fin, fout, fobs, str(steps), str(grid)], capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    out = np.fromfile(fout, dtype=np.float32)
    obs = np.fromfile(fobs).reshape(len(cases), steps + 1, 11)
    off = 0
    for i, c in enumerate(cases):
        nx, npp = shape(c)[:2]
        W = out[off:off + nx * npp].reshape(npp, nx)
        off += nx * npp
        ref_obs, ref = WignerOracle(params(c)).run(W0[i], steps)
        # measured: FP32 2.4e-7 .. 3.1e-7 (state), 2.6e-7 .. 2.8e-6 (energy); mixed 5e-8 .. 2.3e-7
        # (state, FP32 storage rounding), 7e-10 .. 8e-9 (energy)
        assert rel_l2(W, ref) < (2e-6 if prec == 0 else 5e-7), (i, rel_l2(W, ref))
        assert np.max(np.abs(obs[i, :, 0] - ref_obs[:, 0])) < (1e-6 if c['gamma'] else 2e-8 * steps), i
        assert np.max(np.abs(obs[i, :, 1:10] - ref_obs[:, 1:10])) < 1e-4, i
        assert np.max(np.abs(obs[i, :, 9] - ref_obs[:, 9])) < (1e-5 if prec == 0 else 3e-8), i


@pytest.mark.parametrize('prec,gamma', [(0, 0.), (1, 0.1)])
def test_adjoint_device_code_matches_twin(staged, prec, gamma):
    """The adjoint form on a 128 x 64 grid, 3 steps with controls eps_n, undamped in complex64
    and damped (Caldeira-Leggett order 3 + normalisation) in complex128: the forward against the
    complex128 torch twin, and the adjoint sweep's dL/dW_0, dL/deps_n and dL/d(v4, v2) of
    L = Re <L, W_N> against the twin's autograd."""
    import torch
    from adjoint_twin import Twin
    nx, npp, steps, amp, dt, dth, dla, v4, v2, v0 = 128, 64, 3, 10., 0.005, 0.02, 0.001, 0.05, -1., 0.
    exe = build(staged, 'adjoint_emu.cpp', dict(WIGA_NX=nx, WIGA_NP=npp, WIGA_PW=1, WIGA_PREC=prec))
    cdt = np.complex64 if prec == 0 else np.complex128
    rng = np.random.default_rng(4)
    eps = rng.normal(0., 0.3, steps)
    dx, dp = 2 * amp / nx, 2 * amp / npp
    xg = (dx * np.fft.fftshift(np.arange(nx) - nx // 2))[None, :]
    pg = (dp * np.fft.fftshift(np.arange(npp) - npp // 2))[:, None]
    X = np.exp(-((xg + 1.5) ** 2 + (pg - 0.4) ** 2)).astype(cdt)
    L = (rng.normal(size=(npp, nx)) + 1j * rng.normal(size=(npp, nx))).astype(cdt)
    names = ('a_x.bin', 'a_l.bin', 'a_eps.bin', 'a_w.bin', 'a_lam.bin', 'a_grad.bin')
    fx, fl, fe, fw, flam, fg = (os.path.join(staged, n) for n in names)
    X.tofile(fx)
    L.tofile(fl)
    eps.tofile(fe)
    r = subprocess.run([exe, fx, fl, fe, fw, flam, fg, str(steps)] +
                       [repr(v) for v in (amp, dt, dth, dla, v4, v2, v0, gamma, 0.)],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    W = np.fromfile(fw, dtype=cdt).reshape(npp, nx).astype(np.complex128)
    lam = np.fromfile(flam, dtype=cdt).reshape(npp, nx).astype(np.complex128)
    grad = np.fromfile(fg).reshape(steps, 3)
    tw = Twin(nx, npp, amp, dt, d_theta=dth, d_lambda=dla, v4=v4, v2=v2, v0=v0, gamma=gamma)
    X128 = torch.from_numpy(X.astype(np.complex128)).requires_grad_(True)
    L128 = torch.from_numpy(L.astype(np.complex128))
    e128 = torch.tensor(eps, requires_grad=True)
    coef = torch.tensor([v4, v2], dtype=torch.float64, requires_grad=True)
    WT = tw.propagate(X128, e128, coef)
    assert rel_l2(W, WT.detach().numpy()) < (1e-5 if prec == 0 else 1e-13), rel_l2(W, WT.detach().numpy())
    torch.real(torch.vdot(L128.flatten(), WT.flatten())).backward()
    tol = 2e-5 if prec == 0 else 1e-11
    assert rel_l2(lam, X128.grad.numpy()) < tol, rel_l2(lam, X128.grad.numpy())
    ge = e128.grad.numpy()
    assert np.linalg.norm(grad[:, 0] - ge) < tol * np.linalg.norm(ge), (grad[:, 0], ge)
    gc = grad[:, 1:].sum(axis=0)
    ctol = 1e-4 if prec == 0 else 1e-11    # FP32: measured 2.4e-5 for dL/dv4 (weights ~x u (x^2 + u^2))
    assert np.all(np.abs(gc - coef.grad.numpy()) < ctol * np.abs(coef.grad.numpy())), (gc, coef.grad)


# imaginary-time (Bloch) steps, GPU_Wigner2D_GPitaevskii_Bloch: the ground-state iteration with the
# mean-field term, and the excited-state one (projection on W0) without it
@pytest.mark.parametrize('a_gp,with_w0', [(0.5, False), (0., True)])
def test_bloch_device_code_matches_oracle(staged, a_gp, with_w0):
    from oracle.gpitaevskii import BlochOracle
    exe = build(staged, 'wigner2d_emu.cpp', dict(WIG_NX=WNX, WIG_NP=WNP, WIG_XROWS=4, WIG_XNT=32,
                                                 WIG_KIN_STRING=1, WIG_PC=8, WIG_PNT=32, WIG_DAMP=1,
                                                 WIG_RNT=256, WIG_XMINB=1, WIG_PMINB=1, WIG_STRANG=1))
    prm = WignerParams(WNX, WNP, WXA, WPA, WDT, potential=WPOT, dpotential=WDPOT, kinetic='0.5*p*p',
                       constants='exact')
    orc = BlochOracle(prm, a_gp)
    X = np.fft.fftshift(np.linspace(-WXA, WXA - 2 * WXA / WNX, WNX))[np.newaxis, :]
    P = np.fft.fftshift(np.linspace(-WPA, WPA - 2 * WPA / WNP, WNP))[:, np.newaxis]
    W = orc.initial_normalise(np.exp(-(X - 1.5) ** 2 - (P + 0.5) ** 2 * 1.3) + 0. * 1j)
    W0 = orc.initial_normalise(np.exp(-(X + 0.5) ** 2 - P ** 2) + 0. * 1j) if with_w0 else None
    steps, dtb = 2, WDT
    fin, fout, fst, fw0 = (os.path.join(staged, n) for n in ('bl_in.bin', 'bl_out.bin', 'bl_st.bin', 'bl_w0.bin'))
    W.tofile(fin)
    if with_w0:
        W0.tofile(fw0)
    r = subprocess.run([exe, fin, fout, fst, '1'] + [repr(v) for v in (WXA, WPA, WDT, 0., 0., 0.)] +
                       ['0', repr(a_gp), str(steps), repr(dtb), fw0 if with_w0 else '-'],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = np.fromfile(fout, dtype=np.complex128).reshape(WNP, WNX)
    st = np.fromfile(fst).reshape(steps, 10)
    for k in range(steps):
        W = orc.step_bloch(W, k * WDT, dtb, W0)
        out, purity, nle = orc.stats(W)
        ref = np.array([v.real for v in out] + [purity.real, purity.imag, np.real(nle)])
        got_k = np.concatenate([st[k, :7], st[k, 7:8]])
        assert np.all(np.abs(got_k - ref) <= 1e-10 * np.maximum(np.abs(ref), 1e-3)), (k, got_k - ref)
        if with_w0:
            assert st[k, 8] == float(np.any(W.sum(axis=1).real * prm.dX < 0.))
    assert rel_l2(got, W) < 1e-12
