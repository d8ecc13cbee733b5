"""pytest configuration: the ``gpu`` marker and shared fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


# WIG_CPU_FULL=1 adds the heavier CPU parametrisations (more sanitizer runs, more
# NVRTC compiles of the batched module, larger host executions of the device
# code); the default CPU suite keeps one representative of each to a few minutes.
FULL = os.environ.get('WIG_CPU_FULL', '') == '1'


def full_only(*values):
    """A pytest.param that runs only with WIG_CPU_FULL=1."""
    return pytest.param(*values, marks=pytest.mark.skipif(not FULL, reason='WIG_CPU_FULL=1 runs it'))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a)')


@pytest.fixture(scope='session')
def golden_dir():
    return os.path.join(ROOT, 'tests', 'golden')
