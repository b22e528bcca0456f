"""Test configuration: the `gpu` marker, and imports of the package (openmm-lbm_b200/, imported as lbm_b200) and
of the CPU oracles (oracle/oracle.py, test infrastructure)."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load_package():
    if 'lbm_b200' in sys.modules:
        return sys.modules['lbm_b200']
    path = os.path.join(ROOT, 'openmm-lbm_b200')
    spec = importlib.util.spec_from_file_location('lbm_b200', os.path.join(path, '__init__.py'),
                                                  submodule_search_locations=[path])
    module = importlib.util.module_from_spec(spec)
    sys.modules['lbm_b200'] = module
    spec.loader.exec_module(module)
    return module


_load_package()
sys.path.insert(0, os.path.join(ROOT, 'oracle'))
sys.path.insert(0, os.path.join(ROOT, 'tests'))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200)')


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason='no CUDA device')
    for item in items:
        if 'gpu' in item.keywords:
            item.add_marker(skip)


@pytest.fixture(autouse=True)
def _release_kernels():
    """Destroy the kernels and device objects a test leaves behind while the test session is still running, so that
    none is finalized during interpreter shutdown."""
    yield
    import gc
    gc.collect()
