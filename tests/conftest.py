"""Shared fixtures.  Tests marked `gpu` need a CUDA device (B200); everything
else runs on CPU.  The oracle (oracle/) is test infrastructure: the numpy
restatement always, the compiled reference (oracle/_ref) when it has been
built (`make -C oracle`, needs the reference sources)."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running parity case")


@pytest.fixture(scope="session")
def cf():
    return importlib.import_module("ubiquitous-spoon_b200")


@pytest.fixture(scope="session")
def ref():
    import ref as ref_mod
    if not ref_mod.available():
        if os.path.isdir(ref_mod.REFERENCE_SRC):
            ref_mod.build()
        else:
            pytest.skip("compiled reference (oracle/_ref) not available")
    return ref_mod


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.cuda.get_device_name(0)
