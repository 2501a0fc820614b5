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
    config.addinivalue_line("markers", "refjob(name): uses the reference run `name` of tests/ref_jobs.py")


_jobs = None


def _jobset():
    global _jobs
    if _jobs is None:
        import tempfile
        import ref_jobs
        base = os.environ.get("CF_REFJOB_DIR") or None
        _jobs = ref_jobs.JobSet(tempfile.mkdtemp(prefix="cf_refjobs_", dir=base))
    return _jobs


def pytest_collection_finish(session):
    """Start the reference runs that the selected tests need, in child
    processes, before any test (and any GPU work) runs."""
    import ref as ref_mod
    if session.config.option.collectonly:
        return
    names = []
    for item in session.items:
        m = item.get_closest_marker("refjob")
        if m is not None and m.args[0] not in names:
            names.append(m.args[0])
    if names and ref_mod.available():
        js = _jobset()
        for n in names:
            js.start(n)


def pytest_sessionfinish(session, exitstatus):
    global _jobs
    if _jobs is not None:
        import shutil
        _jobs.stop()
        shutil.rmtree(_jobs.folder, ignore_errors=True)
        _jobs = None


@pytest.fixture(scope="session")
def refjobs(ref):
    return _jobset()


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
