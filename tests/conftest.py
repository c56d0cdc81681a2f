"""Test setup: the ``gpu`` marker and import paths.

``cutile`` (the product) lives in ``cutile-stencil-dsl_b200/``; the oracle
in ``oracle/``; test helpers in ``tests/``.
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "cutile-stencil-dsl_b200"), ROOT, os.path.dirname(__file__)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    path = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def golden_exprs():
    import json

    with open(os.path.join(os.path.dirname(__file__), "golden", "golden_exprs.json")) as f:
        return json.load(f)
