"""Shared test setup: import paths, the gpu marker, and built artefacts.

`-m "not gpu"` runs on a machine without a GPU (oracle, plan compiler, file
format, generators, C-ABI exports, multi-process logic over gloo).
`-m gpu` tests call the CUDA path through the C-ABI and compare it with the
oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the product library and the oracle once per session."""
    from pumatch_b200 import build as pmbuild
    pmbuild.build()
    import pm_oracle
    pm_oracle.build()
    yield


@pytest.fixture(scope="session")
def ctx():
    import pumatch_b200 as pm
    c = pm.Context(0)
    yield c
    c.close()
