"""Shared pytest setup: import paths, the ``gpu`` marker, fixture helpers."""

import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "jax-mtp_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")
POTENTIALS = os.path.join(GOLDEN, "potentials")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden_case(tag):
    z = np.load(os.path.join(GOLDEN, f"phys_{tag}.npz"), allow_pickle=False)
    return {k: z[k] for k in z.files}


def potential_path(name):
    return os.path.join(POTENTIALS, name)


@pytest.fixture(scope="session")
def cuda_available():
    import torch
    return torch.cuda.is_available()
