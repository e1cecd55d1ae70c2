"""Test configuration: the `gpu` marker and shared fixtures.

`-m "not gpu"` runs on a machine without a GPU (oracle known-answer tests,
model compiler, host logic, C-ABI exports); `-m gpu` runs the CUDA backend
against the oracle on a B200.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# checkout of the reference repository, for the tests that read its files;
# unset: those tests use the committed fixtures under tests/golden/ instead
REFERENCE = os.environ.get("PIPPIN_REFERENCE", "")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built backend library")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    O.build()
    return O


def have_reference():
    return bool(REFERENCE) and os.path.isdir(os.path.join(REFERENCE, "assets"))
