import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _build_native():
    # build.py is loaded by path: importing the package needs the built library
    import importlib.util
    spec = importlib.util.spec_from_file_location("kc_build", os.path.join(ROOT, "kmertreecounter_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build()
    import oracle
    oracle.build()


_build_native()


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)


def has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
