"""The device code's host execution (tests/emu/, see test_emu_cpu.py) under
sanitizers, one run per kernel family:

* ThreadSanitizer: every CUDA thread is a host thread and __syncthreads /
  __syncwarp are std::barrier waits, so a shared-memory (or global) access by
  one thread that no barrier orders against another thread's write of the
  same address -- a missing or misplaced barrier -- is reported as a data race
  and the run exits non-zero;
* AddressSanitizer + UndefinedBehaviorSanitizer: each launch's dynamic shared
  memory is a heap buffer of exactly the size the library passes for it, so an
  index past it is reported, as are heap overflows of the global arrays and
  undefined behaviour.

Every run also has the device code's own index checks (WIG_BOUNDS) on and its
shared memory filled with NaN before each block, and still has to match the
oracle / the twin as in test_emu_cpu.py."""
import pytest

import test_emu_cpu as E
from conftest import FULL
from test_emu_cpu import staged  # noqa: F401  (the module-scoped staging fixture)

CASES = [
    ('test_batch_device_code_matches_oracle', dict(warps=4, grid=3, prec=0, xstage=1)),
    ('test_batch_device_code_matches_oracle', dict(warps=2, grid=5, prec=1, xstage=0)),
    ('test_adjoint_device_code_matches_twin', dict(prec=0, gamma=0.)),
    ('test_adjoint_device_code_matches_twin', dict(prec=1, gamma=0.1)),
    ('test_wigner2d_device_code_matches_oracle', dict(xrows=32, xnt=256, pc=64, pnt=256, odm=0, kvn=0)),
    ('test_wigner2d_device_code_matches_oracle', dict(xrows=4, xnt=32, pc=8, pnt=32, odm=2, kvn=0)),
    ('test_strang_gp_device_code_matches_oracle', dict(xrows=4, xnt=32, pc=8, pnt=32, odm=1, a_gp=-0.3)),
    ('test_bloch_device_code_matches_oracle', dict(a_gp=0.5, with_w0=False)),
    ('test_dirac2d_device_code_matches_oracle', dict(rows=4, rnt=64, cc=8, cnt=64)),
    ('test_dirac3d_cubic_planner_tiles', dict(n=16)),
]
# the default CPU suite: the race checker over the batched (mixed, direct x-pass loads), adjoint
# (damped), complex128 Wigner (ODM) and Dirac2D passes, AddressSanitizer over the Dirac2D
# passes; every pair with WIG_CPU_FULL=1 (run before a change to the kernels is committed)
DEFAULT = {('thread', 1), ('thread', 3), ('thread', 5), ('thread', 8), ('address', 8)}


def _ids(case):
    name, kw = case
    return name.replace('test_', '').replace('_device_code_matches_oracle', '').replace(
        '_device_code_matches_twin', '') + '-' + '-'.join('%s' % v for v in kw.values())


@pytest.mark.parametrize('sanitize', ['thread', 'address'])
@pytest.mark.parametrize('case', CASES, ids=[_ids(c) for c in CASES])
def test_device_code_under_sanitizer(staged, monkeypatch, sanitize, case):  # noqa: F811
    if (sanitize, CASES.index(case)) not in DEFAULT and not FULL:
        pytest.skip('WIG_CPU_FULL=1 runs it (the default CPU suite keeps to a few minutes)')
    build = E.build
    monkeypatch.setattr(E, 'build', lambda dst, source, macros: build(dst, source, macros, sanitize=sanitize))
    name, kw = case
    getattr(E, name)(staged, **kw)
