import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a)')


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope='session')
def port():
    from oracle.oracle import Oracle
    return Oracle('port')


@pytest.fixture(scope='session')
def ref():
    from oracle.oracle import Oracle, available
    if not available('ref'):
        pytest.skip('oracle/_ref not built (reference sources absent)')
    return Oracle('ref')


def load_probe():
    """libtb_probe.so (tests/probe): the test and measurement helpers kept
    out of the product library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location('tb_probe_loader', os.path.join(REPO, 'tests', 'probe', 'loader.py'))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.load()


@pytest.fixture(scope='session')
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from traceon_b200 import backend
    return backend
