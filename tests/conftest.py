import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "siam-quantum_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
# The reference source tree (teepanis/siam-quantum) when a test needs its files directly:
# environment variable SQ_REFERENCE; tests that need it are skipped when it is unset.
REFERENCE = os.environ.get("SQ_REFERENCE", "")


def results_path(name):
    """Where a GPU test leaves its measured figures as JSON (directory SQB200_TEST_RESULTS,
    default test_results/ at the repository root, created on first use)."""
    d = os.environ.get("SQB200_TEST_RESULTS", os.path.join(ROOT, "test_results"))
    os.makedirs(d, exist_ok=True)
    return os.path.join(d, name)


def load_sqb200():
    """Import the package directory siam-quantum_b200/ as module `sqb200`."""
    if "sqb200" in sys.modules and hasattr(sys.modules["sqb200"], "JKEngine"):
        return sys.modules["sqb200"]
    spec = importlib.util.spec_from_file_location("sqb200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["sqb200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import port
    return port


def golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: d[k] for k in d.files}


def golden_basis(g):
    """Basis object built from the reference's own genBasis arrays stored in a fixture."""
    sqb = load_sqb200()
    return sqb.basis.Basis(g["nprim"], g["lmn"], g["xyz"], g["exps"], g["coefs"], g["norms"])


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libsqb200.so")


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


GOLDEN_CASES = ["water_321g", "oh_321g_uhf", "h2co_631gs", "benzene_631gs"]
