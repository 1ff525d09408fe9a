"""Shared pytest configuration: repository on sys.path, the ``gpu`` marker and
small seeded scenes used by the parity tests."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REFERENCE = os.environ.get("SOLWEIG_REFERENCE_TREE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "reference: needs the reference source tree (this container)")


def have_reference():
    return os.path.isfile(os.path.join(REFERENCE, "src", "umep_solweig.py"))


@pytest.fixture(scope="session")
def umep():
    if not have_reference():
        pytest.skip("reference tree not present")
    if REFERENCE not in sys.path:
        sys.path.insert(0, REFERENCE)
    import src.umep_solweig as U
    return U


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def small_scene(n=48, seed=3):
    from solweig_cuda_b200 import synthetic
    return synthetic.make_scene(n, seed=seed)
