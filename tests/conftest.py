"""Test configuration: import paths and the ``gpu`` marker.

``-m "not gpu"`` runs on any machine (oracle pins, host logic, library
symbols); ``-m gpu`` needs a CUDA device and calls libpfflip.so.
"""

import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "implementation-of-adaptive-phase-field-flip_b200")
for p in (PKG, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libpfflip.so")


def pytest_collection_modifyitems(config, items):
    import torch

    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np

    d = os.path.join(REPO, "tests", "golden")
    arrays = np.load(os.path.join(d, "golden.npz"))
    meta = json.load(open(os.path.join(d, "golden.json")))
    return arrays, meta
