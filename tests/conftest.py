"""Shared pytest setup: the `gpu` marker, repo root on sys.path, the oracle library built once."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, 'tests', 'golden')
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200) and the built libopensol_fdtd.so')


@pytest.fixture(scope='session', autouse=True)
def oracle_built():
    """Build the oracle's C restatement (gcc) before any test uses it."""
    subprocess.run(['make', '-s', '-C', os.path.join(ROOT, 'oracle')], check=True)


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_available():
        return
    skip = pytest.mark.skip(reason='no CUDA device')
    for item in items:
        if 'gpu' in item.keywords:
            item.add_marker(skip)
